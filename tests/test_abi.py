"""The C-ABI library loads on any host and exports every declared entry point;
without a GPU, context creation fails with a status, never a crash."""
import ctypes
import os

import pytest

from conftest import needs_library

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    from tom_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libtomgpu.so not built")
    return _lib


def test_exports_every_declared_symbol():
    L = _lib()
    names = L.declared_symbols()
    assert len(names) >= 25
    raw = ctypes.CDLL(L.LIB_PATH)
    missing = [n for n in names if not hasattr(raw, n)]
    assert not missing, missing
    # the ctypes binding declares a signature for exactly these entry points
    assert set(L._SIGS) == set(names)


def test_status_strings_and_version():
    L = _lib()
    lib = L.lib()
    assert lib.tomgpu_version().startswith(b"tomgpu")
    for s in range(8):
        assert lib.tomgpu_status_string(s)
    assert lib.tomgpu_status_string(99) == b"unknown status"


def test_null_arguments_rejected_without_device():
    L = _lib()
    lib = L.lib()
    assert lib.tomgpu_ctx_create(0, None) == L.TOMGPU_ERR_ARG
    assert lib.tomgpu_rotate3d(None, None, None, None, None, 1, None) == L.TOMGPU_ERR_ARG
    assert lib.tomgpu_match_run_dev(None, None, 0, 0, None, None) == L.TOMGPU_ERR_ARG
    m = (ctypes.c_float * 9)()
    e = (ctypes.c_float * 3)(0, 0, 0)
    assert lib.tomgpu_euler_matrix(e, m) == 0 and list(m) == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_context_creation_reports_missing_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib()
    h = ctypes.c_void_p()
    st = L.lib().tomgpu_ctx_create(0, ctypes.byref(h))
    assert st == L.TOMGPU_ERR_CUDA and not h.value
    assert b"device" in L.lib().tomgpu_last_error(None)


@needs_library
def test_host_matrix_equals_oracle(oracle):
    """tomgpu_euler_matrix (host C++) equals the oracle's restatement bit for bit."""
    import numpy as np
    import tom_b200
    rng = np.random.default_rng(5)
    for _ in range(200):
        e = rng.choice([0, 30, 45, 60, 90, 135, 270, 330, 12.5, 77.0, 181.25], 3)
        if rng.random() < 0.5:
            e = (rng.random(3) * 360).astype(np.float32)
        assert np.array_equal(tom_b200.euler_matrix(e), oracle.euler_matrix(e))


_NULL_CALLS = r'''
import ctypes, json, sys
sys.path.insert(0, sys.argv[1])
from tom_b200 import _lib
L = _lib.lib()
out = {}
for name, (res, args) in _lib._SIGS.items():
    if res is ctypes.c_char_p:
        continue
    vals = [0 if a in (ctypes.c_int, ctypes.c_int64, ctypes.c_size_t) else
            0.0 if a in (ctypes.c_float, ctypes.c_double) else None for a in args]
    out[name] = getattr(L, name)(*vals)
print(json.dumps(out))
'''


def test_every_entry_point_rejects_null_arguments():
    """Each entry point called with NULL handles and pointers and zero sizes
    returns TOMGPU_ERR_ARG (the destroy calls, like free, accept NULL; the
    counters read 0), and none of them crashes the process.  The calls run in
    a child process so that a crash fails this test instead of the session."""
    import json
    import subprocess
    import sys
    L = _lib()
    p = subprocess.run([sys.executable, "-c", _NULL_CALLS, ROOT], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    got = json.loads(p.stdout.strip().splitlines()[-1])
    accept_null = {"tomgpu_ctx_destroy", "tomgpu_match_plan_destroy"}
    counters = {"tomgpu_ctx_launch_count", "tomgpu_match_plan_bytes"}
    assert set(got) == {n for n in L._SIGS if L._SIGS[n][0] is not ctypes.c_char_p}
    for name, st in got.items():
        if name in accept_null:
            assert st == L.TOMGPU_OK, name
        elif name in counters:
            assert st == 0, name
        else:
            assert st == L.TOMGPU_ERR_ARG, (name, st)
