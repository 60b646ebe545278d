"""Host copies of the library run on the context's own stream.

Each context launches its kernels on a stream created non-blocking, which
does not wait for work on the legacy default stream.  A blocking cudaMemcpy
from pageable host memory runs on that legacy stream and may return before
its DMA lands; a cudaMemset without a stream also runs there.  Either one,
followed by a kernel on the context's stream, lets the kernel read the
buffer before the copy is done.  This scan keeps every host-to-device copy
and every memset of the library on an explicit stream.  The self-test is the
one exception: its memsets and its kernel all run on the legacy stream."""
import pathlib
import re

CSRC = pathlib.Path(__file__).resolve().parents[1] / "scadyn_b200" / "csrc"
LEGACY_OK = {"selftest.cu"}


def _calls(text, name):
    """(line, argument text) of every call of `name` in text."""
    out = []
    for m in re.finditer(r"\b%s\s*\(" % re.escape(name), text):
        depth, i = 1, m.end()
        while depth and i < len(text):
            depth += {"(": 1, ")": -1}.get(text[i], 0)
            i += 1
        out.append((text.count("\n", 0, m.start()) + 1, text[m.end():i - 1]))
    return out


def _sources():
    files = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h"))
    assert files, CSRC
    return files


def test_no_blocking_host_to_device_copies():
    bad = []
    for f in _sources():
        text = f.read_text()
        for name in ("cudaMemcpy", "cudaMemcpyToSymbol"):
            for line, args in _calls(text, name):
                if "HostToDevice" in args or name == "cudaMemcpyToSymbol":
                    bad.append(f"{f.name}:{line} {name}({args[:60]})")
    assert not bad, "blocking host-to-device copies on the legacy stream:\n" + "\n".join(bad)


def test_no_legacy_stream_memsets():
    bad = []
    for f in _sources():
        if f.name in LEGACY_OK:
            continue
        for line, args in _calls(f.read_text(), "cudaMemset"):
            bad.append(f"{f.name}:{line} cudaMemset({args[:60]})")
    assert not bad, "memsets on the legacy stream:\n" + "\n".join(bad)


def test_scan_finds_a_planted_copy():
    text = "int f(ctx *c) {\n  cudaMemcpy(d, h.data(), n, cudaMemcpyHostToDevice);\n  cudaMemset(p, 0, 4);\n}\n"
    assert _calls(text, "cudaMemcpy") == [(2, "d, h.data(), n, cudaMemcpyHostToDevice")]
    assert _calls(text, "cudaMemset") == [(3, "p, 0, 4")]
    assert _calls(text, "cudaMemcpyAsync") == []
