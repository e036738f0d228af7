"""CPU checks of the C ABI: the library loads, exports every entry point that
include/gsr.h declares, and the ctypes structure layouts match the header
(sizes and offsets printed by a C program compiled against it)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "gsr.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gsr_[a-z0-9_]+)\s*\(", text)))


def test_header_functions_listed_in_binding():
    from rustscan_b200 import _lib

    assert declared_functions() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    from rustscan_b200 import _lib

    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libgsr.so not built")
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True)
    syms = set(line.split()[-1] for line in out.stdout.splitlines() if line.strip())
    missing = [f for f in declared_functions() if f not in syms]
    assert not missing, missing
    L = _lib.load()  # loads without a GPU; no compute call is made
    assert L.gsr_version().decode().startswith("gsr")


def test_struct_layouts_match_header():
    from rustscan_b200 import _lib

    structs = {
        "gsr_config": _lib.gsr_config,
        "gsr_camera": _lib.gsr_camera,
        "gsr_splats": _lib.gsr_splats,
        "gsr_grads": _lib.gsr_grads,
        "gsr_adam_state": _lib.gsr_adam_state,
        "gsr_lr": _lib.gsr_lr,
        "gsr_train_params": _lib.gsr_train_params,
        "gsr_tune_candidate": _lib.gsr_tune_candidate,
        "gsr_tune_result": _lib.gsr_tune_result,
        "gsr_topo_row": _lib.gsr_topo_row,
        "gsr_topo_params": _lib.gsr_topo_params,
        "gsr_frame": _lib.gsr_frame,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{name}.{fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        open(src, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c99", src, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(line.split() for line in out if line.strip())
    for name, cls in structs.items():
        assert int(got[name]) == C.sizeof(cls), name
        for fname, _ in cls._fields_:
            assert int(got[f"{name}.{fname}"]) == getattr(cls, fname).offset, f"{name}.{fname}"


def test_product_does_not_import_oracle():
    """The package never reaches the oracle; only tests, smoke and the bench's CPU baseline do."""
    pkg = os.path.join(ROOT, "rustscan_b200")
    pat = re.compile(r"^\s*(from\s+oracle|import\s+oracle|#\s*include\s*[<\"].*oracle)|liboracle", re.M)
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".h", ".cuh", ".cpp")):
                text = open(os.path.join(dirpath, f)).read()
                assert not pat.search(text), f


def test_context_refuses_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rustscan_b200 import Context

    with pytest.raises(RuntimeError):
        Context(max_splats=16)


def _header_signatures():
    """{function: argument count} and {struct: [field names]} from include/gsr.h."""
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    funcs = {}
    for name, args in re.findall(r"\b(gsr_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        a = args.strip()
        funcs[name] = 0 if a in ("", "void") else a.count(",") + 1
    structs = {}
    for body, name in re.findall(r"typedef struct \w+\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            # "uint32_t tile_w, tile_h" declares two fields; arrays keep their name.
            head, *rest = decl.split(",")
            fields.append(re.findall(r"(\w+)\s*(?:\[[^\]]*\])?\s*$", head)[0])
            fields += [re.sub(r"\[.*", "", r).strip().lstrip("*") for r in rest]
        structs[name] = fields
    return funcs, structs


def test_integration_rust_binding_matches_header():
    """INTEGRATION.md's gsr-sys block declares every function of the header
    with the same number of arguments, and every structure with the same
    fields in the same order."""
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = re.search(r"```rust\n(.*?)```", doc, flags=re.S).group(1)
    funcs, structs = _header_signatures()
    rust_funcs = {}
    for name, args in re.findall(r"pub fn (gsr_\w+)\s*\((.*?)\)\s*(?:->[^;]*)?;", block, flags=re.S):
        a = args.strip().rstrip(",")
        rust_funcs[name] = 0 if not a else a.count(":")
    assert sorted(rust_funcs) == sorted(funcs), set(rust_funcs) ^ set(funcs)
    for name, n in funcs.items():
        assert rust_funcs[name] == n, (name, rust_funcs[name], n)
    rust_structs = {}
    for name, body in re.findall(r"pub struct (gsr_\w+)\s*\{(.*?)\}", block, flags=re.S):
        rust_structs[name] = re.findall(r"pub (\w+)\s*:", body)
    for name, fields in structs.items():
        assert name in rust_structs, name
        assert rust_structs[name] == fields, (name, rust_structs[name], fields)
