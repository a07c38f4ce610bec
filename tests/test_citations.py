"""Citations of the reference (file:line) in the committed sources and docs.

Every C-ABI declaration in include/*.h names the reference interface it
replaces or says that it has no counterpart; and, where the reference
sources are present, every line range cited in the sources and the profile
summaries lies inside the cited file."""
import os
import re
import subprocess
from pathlib import Path

import pytest

from cfdtest import ROOT

REF = Path(os.environ.get("CFD_REFERENCE_DIR") or ROOT.parent / "reference")
CITE = re.compile(r"([A-Za-z_0-9]+\.(?:hpp|cpp)):(\d+)(?:-(\d+))?")
DECL = re.compile(r"^(?:int|double|void|const char\*|size_t)\s+(cfd_[a-z_0-9]+)\s*\(")


def _comment_block(lines, i):
    """The declaration's own comment: contiguous lines above it."""
    block = []
    j = i - 1
    while j >= 0 and lines[j].strip() and not lines[j].startswith("}"):
        block.append(lines[j])
        j -= 1
    return "\n".join(reversed(block))


def test_every_declaration_cites_the_reference():
    missing = []
    for h in sorted((ROOT / "include").glob("*.h")):
        lines = h.read_text().splitlines()
        for i, line in enumerate(lines):
            m = DECL.match(line)
            if not m:
                continue
            txt = _comment_block(lines, i)
            if not (CITE.search(txt) or re.search(r"[Nn]o counterpart", txt)):
                missing.append(f"{h.name}:{i + 1} {m.group(1)}")
    assert not missing, missing


@pytest.mark.skipif(not REF.exists(), reason="reference sources absent")
def test_cited_line_ranges_exist():
    index = {}
    for p in REF.rglob("*"):
        if p.suffix in (".hpp", ".cpp") and p.is_file():
            index.setdefault(p.name, []).append(len(p.read_text(errors="replace").splitlines()))
    r = subprocess.run(["git", "ls-files"], cwd=ROOT, capture_output=True, text=True)
    if r.returncode == 0:
        files = r.stdout.split()
    else:  # a copy without git history: the source trees, without their build outputs
        trees = ("cfd-art_b200", "include", "oracle", "tests", "profiles")
        files = [str(p.relative_to(ROOT)) for t in trees for p in (ROOT / t).rglob("*") if p.is_file()]
        files += [p.name for p in ROOT.glob("*.py")]
        build = ("cfd-art_b200/lib/", "oracle/_ref/", "oracle/_build/")
        files = [f for f in files if not f.startswith(build) and "/." not in "/" + f]
    bad = []
    for f in files:
        source = f.endswith((".py", ".cu", ".cuh", ".h", ".cpp", ".c", ".hpp"))
        if not (source or (f.startswith("profiles/") and f.endswith(".md"))):
            continue
        for ln, line in enumerate((ROOT / f).read_text(errors="replace").splitlines(), 1):
            for m in CITE.finditer(line):
                name, a = m.group(1), int(m.group(2))
                b = int(m.group(3) or a)
                if name not in index:
                    bad.append(f"{f}:{ln} {m.group(0)}: no such reference file")
                elif b < a or not any(b <= n for n in index[name]):
                    bad.append(f"{f}:{ln} {m.group(0)}: past the end of the file")
    assert not bad, bad
