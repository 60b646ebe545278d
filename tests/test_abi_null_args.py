"""Error behaviour of the C ABI without a context: every entry point given a
NULL context (or server), NULL pointers and zero sizes returns SCD_BAD_ARG
instead of crashing, destroying NULL is a no-op, and the error-text getters
name the missing object.  A Fortran host that calls before scd_create succeeded, or
after it failed, gets a status to test, as the reference's routines return
to their callers.  The calls run in a child process, so a crash fails this
test instead of ending the run; none of them reaches the GPU."""
import json
import subprocess
import sys

from scadyn_b200 import api, server

CHILD = r"""
import ctypes as C, json, sys
sys.path.insert(0, sys.argv[1])
from scadyn_b200 import api, server
out = {}
for name in api.EXPORTS + server.EXPORTS:
    if name == "scd_selftest_waits":   # takes a device, not a context (tests/test_failure.py)
        continue
    lib = server._lib() if name in server.EXPORTS else api.load_library()
    f = getattr(lib, name)
    args = [0.0 if t is C.c_double else 0 if t in (C.c_int32, C.c_int64, C.c_int) else None
            for t in (f.argtypes or [])]
    r = f(*args)
    out[name] = r.decode() if isinstance(r, bytes) else r
print(json.dumps(out))
"""


def _returns():
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-c", CHILD, root], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_null_context_calls_return_status():
    ret = _returns()
    assert set(ret) == set(api.EXPORTS + server.EXPORTS) - {"scd_selftest_waits"}
    no_op = {"scd_destroy", "scd_server_destroy"}
    text = {"scd_last_error": "null context", "scd_server_error": "null server"}
    counts = {"scd_nearzone_count", "scd_nearzone_bytes"}
    for name, r in ret.items():
        if name in no_op:
            assert r == api.SCD_OK, name
        elif name in text:
            assert r == text[name], (name, r)
        elif name in counts:
            assert r == -1, (name, r)
        else:
            assert r == api.SCD_BAD_ARG, (name, r)
