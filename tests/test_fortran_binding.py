"""The Fortran module scadyn_b200/fortran/scadyn_gpu.f90 against the C headers.

No Fortran compiler is needed: both sides are parsed as text.  Every entry
point of include/*.h must have a bind(C) interface of the same name whose
dummies match the C parameters position by position (a C scalar is a `value` dummy of
the interoperable kind; a C pointer is either a by-reference dummy of the
pointee's kind or a `type(c_ptr), value` address), with the matching result
kind; every C struct the entry points pass must have a bind(C) type with the
same members in the same order and kinds, so the two layouts agree.
"""
import pathlib
import re

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent
F90 = ROOT / "scadyn_b200" / "fortran" / "scadyn_gpu.f90"
HEADERS = sorted((ROOT / "include").glob("*.h"))

# C scalar type -> Fortran kind spelling
C_SCALAR = {
    "int": "integer(c_int)",
    "int32_t": "integer(c_int32_t)",
    "int64_t": "integer(c_int64_t)",
    "double": "real(c_double)",
    "float": "real(c_float)",
    "scd_c128": "complex(c_double_complex)",
    "scd_c64": "complex(c_float_complex)",
}


def _strip_c_comments(s):
    return re.sub(r"/\*.*?\*/", "", s, flags=re.S)


def c_prototypes():
    out = {}
    for h in HEADERS:
        src = _strip_c_comments(h.read_text())
        for m in re.finditer(r"SCD_API\s+([^;(]*?)\b(scd_\w+)\s*\(([^)]*)\)\s*;", src):
            ret, name, args = m.group(1).strip(), m.group(2), m.group(3)
            params = []
            for a in args.split(","):
                a = " ".join(a.split())
                if not a or a == "void":
                    continue
                stars = a.count("*")
                toks = a.replace("*", " ").replace("const", " ").split()
                params.append((toks[-2], stars, toks[-1]))
            out[name] = (ret.replace("const", "").strip(), params)
    return out


def c_structs():
    out = {}
    for h in HEADERS:
        src = _strip_c_comments(h.read_text())
        for m in re.finditer(r"typedef struct (\w+)\s*\{(.*?)\}\s*(\w+)\s*;", src, flags=re.S):
            members = []
            for decl in m.group(2).split(";"):
                decl = " ".join(decl.replace("const", " ").split())
                if not decl:
                    continue
                ptr = "*" in decl
                head, names = decl.replace("*", " ").split(None, 1)
                for nm in names.split(","):
                    nm = nm.strip()
                    dim = 1
                    am = re.match(r"(\w+)\[(\d+)\]", nm)
                    if am:
                        nm, dim = am.group(1), int(am.group(2))
                    members.append((nm.lower(), "ptr" if ptr else head, dim))
            out[m.group(3)] = members
    return out


def _fortran_statements():
    """Statements of the module with comments removed and & continuations joined."""
    text = []
    for line in F90.read_text().splitlines():
        line = line.split("!", 1)[0].rstrip()
        text.append(line)
    joined, acc = [], ""
    for line in text:
        s = line.strip()
        if acc:
            s = s.lstrip("&").strip()
        if s.endswith("&"):
            acc += s[:-1] + " "
            continue
        joined.append(acc + s)
        acc = ""
    return [s for s in joined if s]


def _decl(stmt):
    """`<type-spec>[, attrs] :: names` -> (kind spelling, attrs, [(name, dim)])."""
    lhs, rhs = stmt.split("::", 1)
    parts = [p.strip().lower() for p in re.split(r",(?![^()]*\))", lhs)]
    kind, attrs = parts[0].replace(" ", ""), set(parts[1:])
    names = []
    for nm in re.split(r",(?![^()]*\))", rhs):
        nm = nm.split("=", 1)[0].strip().lower()
        dm = re.match(r"(\w+)\((\d+|\*)\)", nm)
        if dm:
            names.append((dm.group(1), dm.group(2)))
        else:
            names.append((nm, None))
    return kind, attrs, names


def fortran_interfaces():
    out, cur = {}, None
    for s in _fortran_statements():
        m = re.match(r"(.*?)\bfunction\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*C\s*,\s*name\s*=\s*\"(\w+)\"\s*\)", s, re.I)
        if m:
            cur = {
                "result": m.group(1).strip().lower().replace(" ", ""),
                "dummies": [d.strip().lower() for d in m.group(3).split(",") if d.strip()],
                "decl": {},
            }
            out[m.group(4)] = cur
            continue
        if cur is not None and re.match(r"end\s+function", s, re.I):
            cur = None
            continue
        if cur is not None and "::" in s and not s.lower().startswith("import"):
            kind, attrs, names = _decl(s)
            for nm, dim in names:
                cur["decl"][nm] = (kind, attrs, dim)
    return out


def fortran_types():
    out, cur = {}, None
    for s in _fortran_statements():
        m = re.match(r"type\s*,\s*bind\s*\(\s*C\s*\)[^:]*::\s*(\w+)", s, re.I)
        if m:
            cur = out.setdefault(m.group(1), [])
            continue
        if cur is not None and re.match(r"end\s+type", s, re.I):
            cur = None
            continue
        if cur is not None and "::" in s:
            kind, _, names = _decl(s)
            for nm, dim in names:
                cur.append((nm, kind, int(dim) if dim and dim != "*" else 1))
    return out


def test_every_entry_point_is_bound():
    protos, ifaces = c_prototypes(), fortran_interfaces()
    assert len(protos) >= 30
    missing = sorted(set(protos) - set(ifaces))
    assert not missing, f"entry points without a Fortran interface: {missing}"
    public = " ".join(s for s in _fortran_statements() if s.lower().startswith("public ::")).lower()
    for name in protos:
        if name in ("scd_last_error", "scd_server_error"):
            assert name + "_f" in public, f"{name}: no public Fortran-string wrapper"
        else:
            assert re.search(rf"\b{name.lower()}\b", public), f"{name} is not public"


@pytest.mark.parametrize("name", sorted(c_prototypes()))
def test_interface_matches_prototype(name):
    ret, params = c_prototypes()[name]
    f = fortran_interfaces()[name]
    rk = "type(c_ptr)" if "*" in ret or ret == "char" else C_SCALAR[ret]
    assert f["result"] == rk, f"{name}: result {f['result']} for C {ret}"
    assert len(f["dummies"]) == len(params), f"{name}: {len(f['dummies'])} dummies for {len(params)} parameters"
    for dummy, (ctype, stars, cname) in zip(f["dummies"], params):
        kind, attrs, dim = f["decl"][dummy]
        where = f"{name}({dummy})"
        if stars == 0:
            assert "value" in attrs, f"{where}: C scalar passed by value needs VALUE"
            assert kind == C_SCALAR[ctype], f"{where}: {kind} for C {ctype}"
        elif kind == "type(c_ptr)" and "value" in attrs:
            assert stars == 1, f"{where}: an address stands for a single pointer"
        elif kind == "type(c_ptr)" and dim == "*":
            # an array of addresses (scd_ctx *const *, scd_c128 *const *): one c_ptr per element
            assert stars == 2 and "intent(in)" in attrs, f"{where}: array of c_ptr"
        elif kind == "type(c_ptr)":
            # the address of an opaque handle (scd_ctx **, scd_server **)
            assert stars == 2 and "intent(out)" in attrs, f"{where}: c_ptr by reference"
        else:
            assert stars == 1 and "value" not in attrs, f"{where}: pointer dummy passed by reference"
            want = C_SCALAR.get(ctype, f"type({ctype})")
            assert kind == want, f"{where}: {kind} for C {ctype} *"


def test_structs_match():
    cs, fs = c_structs(), fortran_types()
    passed = {"scd_grid_desc", "scd_solve_opts", "scd_timing", "scd_request", "scd_server_stats", "scd_tuning"}
    assert passed <= set(cs)
    for name in passed:
        assert name in fs, f"no bind(C) type {name}"
        cm, fm = cs[name], fs[name]
        assert [m[0] for m in fm] == [m[0] for m in cm], f"{name}: member order {fm} vs {cm}"
        for (nm, ct, cdim), (_, fk, fdim) in zip(cm, fm):
            want = "type(c_ptr)" if ct == "ptr" else C_SCALAR.get(ct, f"type({ct})")
            assert fk == want and fdim == cdim, f"{name}.{nm}: {fk}({fdim}) for C {ct}[{cdim}]"


def test_request_carries_solve_options_by_value():
    """scd_request embeds scd_solve_opts: the Fortran type nests it the same way."""
    fm = dict((m[0], m[1]) for m in fortran_types()["scd_request"])
    assert fm["opts"] == "type(scd_solve_opts)"
