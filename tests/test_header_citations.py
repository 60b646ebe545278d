"""Every entry point declared in include/*.h says which reference routine it
replaces (a src/*.f90 file and line range in the comment above it, shared by
a group of declarations), or that it has no counterpart in the reference.
The server header states once, at its top, that its whole layer has no
counterpart."""
import pathlib
import re

INCLUDE = pathlib.Path(__file__).resolve().parents[1] / "include"
CITES = re.compile(r"\.f90:\d+|[Nn]o counterpart")


def _declarations(text):
    """(name, the comment block closest above the declaration)."""
    out = []
    for m in re.finditer(r"SCD_API\s+[^;(]*?\b(scd_\w+)\s*\(", text):
        before = text[:m.start()]
        start, end = before.rfind("/*"), before.rfind("*/")
        out.append((m.group(1), before[start:end] if 0 <= start < end else ""))
    return out


def test_every_entry_point_cites_the_reference():
    missing = []
    for f in sorted(INCLUDE.glob("*.h")):
        text = f.read_text()
        head = text[:text.find("#ifndef")]
        whole_file = bool(re.search(r"no counterpart in the reference", head))
        decls = _declarations(text)
        assert decls, f
        for name, comment in decls:
            if not (whole_file or CITES.search(comment)):
                missing.append(f"{f.name}: {name}")
    assert not missing, "entry points without a reference citation:\n" + "\n".join(missing)
