"""Every line citation of a reference file in this repository points inside
that file: `name.wgsl:N`, `name.wgsl:A-B` (and comma lists of those) for the
shaders, and the same for Rust sources cited by a path whose last components
identify one file of the reference (`engine/trainer.rs:179-191`). Runs when
the RustScan checkout is at hand (the directory RUSTSCAN_REFERENCE names, or
a `reference` directory beside this repository) and skips otherwise."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("RUSTSCAN_REFERENCE", os.path.join(os.path.dirname(ROOT), "reference"))
# This repository's own sources and documents (the only files scanned).
SOURCE_DIRS = ("rustscan_b200", "oracle", "include", "tests")
SOURCE_FILES = ("bench.py", "__graft_entry__.py", "README.md", "DESIGN.md", "INTEGRATION.md")
CITE = re.compile(r"((?:[A-Za-z0-9_]+/)*[A-Za-z0-9_]+\.(?:wgsl|rs)):(\d+(?:-\d+)?(?:,\s?\d+(?:-\d+)?)*)")


def _reference_files():
    files = {}
    for dirpath, dirs, names in os.walk(REF):
        dirs[:] = [d for d in dirs if d not in (".git", "target")]
        for n in names:
            if n.endswith((".wgsl", ".rs")):
                full = os.path.join(dirpath, n)
                files[os.path.relpath(full, REF)] = full
    return files


def _resolve(cited, files):
    """The reference files whose path ends with the cited path."""
    return [f for rel, f in files.items() if rel == cited or rel.endswith("/" + cited)]


def _repo_sources():
    for f in SOURCE_FILES:
        if os.path.isfile(os.path.join(ROOT, f)):
            yield os.path.join(ROOT, f)
    for top in SOURCE_DIRS:
        for dirpath, dirs, names in os.walk(os.path.join(ROOT, top)):
            dirs[:] = [d for d in dirs if d not in ("_build", "__pycache__")]
            for n in names:
                if n.endswith((".py", ".cu", ".cuh", ".h", ".cpp", ".md", "Makefile")):
                    yield os.path.join(dirpath, n)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "RustGS")), reason="reference checkout not present")
def test_reference_line_citations_are_in_range():
    files = _reference_files()
    lines = {}
    bad, checked = [], 0
    for path in _repo_sources():
        for ln, text in enumerate(open(path, errors="ignore"), 1):
            for m in CITE.finditer(text):
                cands = _resolve(m.group(1), files)
                # Shader names are unique; a Rust citation is checked when its
                # path names exactly one file.
                if len(cands) != 1:
                    if m.group(1).endswith(".wgsl"):
                        bad.append((os.path.relpath(path, ROOT), ln, m.group(0), "no such shader"))
                    continue
                f = cands[0]
                if f not in lines:
                    lines[f] = sum(1 for _ in open(f, errors="ignore"))
                for part in re.split(r",\s?", m.group(2)):
                    nums = [int(x) for x in part.split("-")]
                    checked += 1
                    if max(nums) > lines[f] or min(nums) < 1 or nums != sorted(nums):
                        bad.append((os.path.relpath(path, ROOT), ln, m.group(0), f"file has {lines[f]} lines"))
    assert checked > 100
    assert not bad, "\n".join(map(str, bad))
