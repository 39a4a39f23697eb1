"""The Rust binding the integration guide at the repository root writes out
(the declarations a user of the reference adds to call this library from
`src/soft_body/mod.rs`) declares every function of include/arphys.h with the
same number of parameters."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _arity(args):
    args = args.strip()
    if args in ("", "void"):
        return 0
    return len([a for a in args.split(",") if a.strip()])


def header_functions():
    text = open(os.path.join(ROOT, "include", "arphys.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(arp_[a-z0-9_]+)\s*\(([^;{}]*?)\)\s*;", text):
        out[m.group(1)] = _arity(m.group(2))
    return out


def rust_declarations():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return [(m.group(1), _arity(m.group(2))) for m in re.finditer(r"pub fn (arp_[a-z0-9_]+)\(([^)]*)\)", text)]


def rust_functions():
    return dict(rust_declarations())


def test_rust_binding_declares_every_header_function():
    h, r = header_functions(), rust_functions()
    assert len(h) > 40
    missing = sorted(set(h) - set(r))
    assert not missing, f"functions of include/arphys.h without a Rust declaration: {missing}"
    extra = sorted(set(r) - set(h))
    assert not extra, f"Rust declarations with no function in include/arphys.h: {extra}"
    wrong = {f: (h[f], r[f]) for f in h if h[f] != r[f]}
    assert not wrong, f"parameter counts differ (header, Rust): {wrong}"


def test_rust_binding_declares_each_function_once():
    """One crate may not declare an extern function twice."""
    names = [n for n, _ in rust_declarations()]
    dup = sorted({n for n in names if names.count(n) > 1})
    assert not dup, f"declared more than once: {dup}"


def _header_structs():
    text = open(os.path.join(ROOT, "include", "arphys.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"typedef struct (arp_\w+)\s*\{(.*?)\}\s*\1\s*;", text, flags=re.S):
        decls = [d.strip() for d in m.group(2).split(";") if d.strip()]
        out[m.group(1)] = sum(len(d.split(",")) for d in decls)  # `uint32_t mat, solid_id;` is two fields
    return out


def _rust_structs():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    return {m.group(1): len(re.findall(r"\bpub\s+\w+\s*:", m.group(2)))
            for m in re.finditer(r"pub struct (arp_\w+)\s*\{(.*?)\}", text, flags=re.S)}


def test_rust_records_have_the_header_fields():
    """Every record of the header has a #[repr(C)] twin in the binding with the
    same number of fields (the field types follow the header line by line)."""
    h, r = _header_structs(), _rust_structs()
    assert len(h) >= 10
    assert sorted(h) == sorted(r), (sorted(set(h) ^ set(r)))
    wrong = {k: (h[k], r[k]) for k in h if h[k] != r[k]}
    assert not wrong, f"field counts differ (header, Rust): {wrong}"
