"""The C ABI library loads without a GPU and exports every declared entry point."""
import ctypes
import os
import re
import subprocess
import sys

import bitz_b200
from bitz_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            text = open(os.path.join(inc, fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names.update(re.findall(r"\b(bitz_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    for name in sorted(names):
        assert hasattr(lib, name), name


def test_binding_covers_every_declared_symbol():
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert declared_symbols() <= bound


def test_errors_are_reported_not_raised():
    lib = _lib.load()
    rc = lib.bitz_post_gkr_prove(None, 7, None, 0, None, None, 100, None, None, None)
    assert rc == 1
    assert b"null" in lib.bitz_last_error()


def _resident_mode(env_updates):
    env = {k: v for k, v in os.environ.items()
           if k not in ("BITZ_RESIDENT_ROUNDS", "CUDA_INJECTION64_PATH")}
    env.update(env_updates)
    code = ("import ctypes, sys; lib = ctypes.CDLL(sys.argv[1]); "
            "print(lib.bitz_resident_rounds())")
    out = subprocess.run([sys.executable, "-c", code, _lib.LIB_PATH], env=env,
                         capture_output=True, text=True, check=True)
    return int(out.stdout.strip())


def test_resident_rounds_follow_the_environment():
    """Kernels that wait for the host are off under an injected CUDA tool
    (a kernel profiler holds the host at each launch) unless forced on."""
    assert _resident_mode({}) == 1
    assert _resident_mode({"CUDA_INJECTION64_PATH": "/opt/tool/libinject.so"}) == 0
    assert _resident_mode({"CUDA_INJECTION64_PATH": ""}) == 1
    assert _resident_mode({"BITZ_RESIDENT_ROUNDS": "0"}) == 0
    assert _resident_mode({"BITZ_RESIDENT_ROUNDS": "1",
                           "CUDA_INJECTION64_PATH": "/opt/tool/libinject.so"}) == 1
    assert _resident_mode({"BITZ_RESIDENT_ROUNDS": "0",
                           "CUDA_INJECTION64_PATH": "/opt/tool/libinject.so"}) == 0
