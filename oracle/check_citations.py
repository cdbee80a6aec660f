#!/usr/bin/env python
"""Checks every reference citation in this repository against the reference's files.

A citation is ``src/<path>.jl:<lines>`` (or ``test/``, ``docs/``, ``benchmark/``),
where <lines> is a comma list of line numbers and ranges (``:149-158,161``).
Each cited file must exist under the reference checkout and every cited line
must lie inside it.  Prints one line per bad citation and exits 1 if there is any.

    python oracle/check_citations.py [--reference /root/reference]

Test infrastructure: it reads the reference's sources, so it runs only where
they are mounted (the CPU test that calls it skips otherwise).
"""

import argparse
import os
import re
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEFAULT_REF = "/root/reference"
CITE = re.compile(r"\b((?:src|test|docs|benchmark)/[A-Za-z0-9_./-]+\.(?:jl|md|toml)):(\d+(?:-\d+)?(?:,\d+(?:-\d+)?)*)")
# this repository's own sources: the package, the kernels, the header, the
# oracle, the tests, the bench and entry points, and the design and integration notes
SOURCE_DIRS = ("boundarylayerdynamics.jl_b200/BoundaryLayerDynamics", "boundarylayerdynamics.jl_b200/csrc",
               "include", "oracle", "tests")
SOURCE_FILES = ("bench.py", "__graft_entry__.py", "DESIGN.md", "INTEGRATION.md", "README.md")
EXTS = (".py", ".cu", ".cuh", ".h", ".md", ".c", ".cpp")


def repo_files(root):
    for d in SOURCE_DIRS:
        base = os.path.join(root, d)
        for f in sorted(os.listdir(base)) if os.path.isdir(base) else ():
            p = os.path.join(base, f)
            if os.path.isfile(p) and f.endswith(EXTS):
                yield p
    for f in SOURCE_FILES:
        p = os.path.join(root, f)
        if os.path.isfile(p):
            yield p


def line_counts(ref):
    cache = {}

    def n(path):
        if path not in cache:
            p = os.path.join(ref, path)
            if not os.path.isfile(p):
                cache[path] = None
            else:
                with open(p, encoding="utf-8", errors="replace") as fh:
                    cache[path] = sum(1 for _ in fh)
        return cache[path]

    return n


def check(root, ref):
    nlines = line_counts(ref)
    bad, total = [], 0
    for fn in repo_files(root):
        with open(fn, encoding="utf-8", errors="replace") as fh:
            text = fh.read()
        for lineno, line in enumerate(text.splitlines(), 1):
            for m in CITE.finditer(line):
                path, spec = m.group(1), m.group(2)
                total += 1
                n = nlines(path)
                where = f"{os.path.relpath(fn, root)}:{lineno}"
                if n is None:
                    bad.append(f"{where}: {path} does not exist")
                    continue
                for part in spec.split(","):
                    a, _, b = part.partition("-")
                    lo, hi = int(a), int(b or a)
                    if not (1 <= lo <= hi <= n):
                        bad.append(f"{where}: {path}:{part} outside 1-{n}")
    return total, bad


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REF)
    args = ap.parse_args()
    if not os.path.isdir(args.reference):
        print(f"reference not found at {args.reference}")
        return 2
    total, bad = check(REPO, args.reference)
    for b in bad:
        print(b)
    print(f"{total} citations, {len(bad)} bad")
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main())
