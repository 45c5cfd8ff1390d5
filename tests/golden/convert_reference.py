"""Mechanical Python 2 -> 3 conversion of the reference's DMRG package.

This is test infrastructure only.  The reference (zhendongli2008/qcmpodmrg) is
Python 2 code; this container has Python 3 and no lib2to3.  The script rewrites
a copy of ``<reference>/source`` into ``baseline/_ref/qcmpodmrg/source`` so that
``tests/golden/make_golden.py`` can import and run the unmodified algorithms to
produce golden fixtures.  The converted copy is git-ignored and never shipped.

Rewrites applied (syntax only, no algorithmic change):
  * tabs expanded to 8 columns (Python 2 tab semantics);
  * ``print x, y`` statements -> ``print(x, y)`` (trailing comma -> ``end=' '``);
  * implicit relative imports -> explicit relative imports;
  * list-returning ``map/filter/zip/range`` and ``reduce``/``basestring`` shims
    injected at module top;
  * ``d.keys()[0]`` -> ``list(d.keys())[0]``; ``dic.values()`` -> list;
  * integer ``/`` at the three places where Python 2 relied on it
    (mpo_dmrg_dotutil.py:278,286, mpo_dmrg_qphys.py:36);
  * ``string.join`` in itools/molinfo.py;
  * ``size > 0`` tests on possibly-empty MPO-bond slices (``None`` in Python 2 compares
    below 0: mpo_dmrg_initQt.py:170,253, mpo_dmrg_kernelQt.py:694,762,1059,1148).

The C library ``ctypes/qsym.c`` is compiled from where it lies with the
reference's own install.sh command into ``baseline/_ref/qcmpodmrg/libs``.

Usage:  python tests/golden/convert_reference.py [--ref REFERENCE_ROOT]
        (default: the environment variable QCMPODMRG_REFERENCE)
"""
import argparse
import io
import os
import re
import shutil
import subprocess
import sys
import tokenize

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
OUT_ROOT = os.path.join(REPO, "baseline", "_ref")

PRELUDE = (
    "import builtins as _py3b\n"
    "from functools import reduce\n"
    "def map(*a): return list(_py3b.map(*a))\n"
    "def filter(*a): return list(_py3b.filter(*a))\n"
    "def zip(*a): return list(_py3b.zip(*a))\n"
    "def range(*a): return list(_py3b.range(*a))\n"
    "basestring = str\n"
)


def _convert_prints(src):
    """Turn print statements into print() calls using the tokenizer."""
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    lines = src.splitlines(keepends=True)
    # edits: list of (row, col, text_insert) ; applied from the back
    edits = []
    prev_sig = None
    for i, t in enumerate(toks):
        if t.type == tokenize.NAME and t.string == "print":
            at_stmt = prev_sig is None or prev_sig.type in (
                tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT, tokenize.NL) or (
                prev_sig.type == tokenize.OP and prev_sig.string in (":", ";"))
            nxt = toks[i + 1]
            if at_stmt and not (nxt.type == tokenize.OP and nxt.string == "("):
                # find end of statement: NEWLINE, or ';' at depth 0, or COMMENT before NEWLINE
                depth = 0
                j = i + 1
                last = t
                while j < len(toks):
                    tj = toks[j]
                    if tj.type == tokenize.OP and tj.string in "([{":
                        depth += 1
                    elif tj.type == tokenize.OP and tj.string in ")]}":
                        depth -= 1
                    if depth == 0 and (tj.type in (tokenize.NEWLINE, tokenize.COMMENT, tokenize.ENDMARKER)
                                       or (tj.type == tokenize.OP and tj.string == ";")):
                        break
                    if tj.type not in (tokenize.NL,):
                        last = tj
                    j += 1
                trailing = last.type == tokenize.OP and last.string == ","
                if last is t:
                    edits.append((t.end[0], t.end[1], t.end[0], t.end[1], "()"))
                else:
                    if trailing:
                        edits.append((last.start[0], last.start[1], last.end[0], last.end[1], ", end=' ')"))
                    else:
                        edits.append((last.end[0], last.end[1], last.end[0], last.end[1], ")"))
                    # replace the whitespace between print and first arg by '('
                    edits.append((t.end[0], t.end[1], nxt.start[0], nxt.start[1], "("))
        if t.type not in (tokenize.COMMENT, tokenize.NL):
            prev_sig = t
    # apply edits back to front
    edits.sort(key=lambda e: (e[0], e[1]), reverse=True)
    lines = [list(l) for l in lines]
    for (r0, c0, r1, c1, text) in edits:
        if r0 == r1:
            l = lines[r0 - 1]
            l[c0:c1] = list(text)
        else:
            l0 = lines[r0 - 1]
            l0[c0:] = list(text)
            for r in range(r0, r1 - 1):
                lines[r] = []
            l1 = lines[r1 - 1]
            l1[:c1] = []
    return "".join("".join(l) for l in lines)


_IMPORT_RE = re.compile(r"^(\s*)import\s+([A-Za-z_][\w\.]*(?:\s*,\s*[A-Za-z_][\w\.]*)*)\s*(#.*)?$")
_FROM_RE = re.compile(r"^(\s*)from\s+([A-Za-z_][\w]*)((?:\.[\w]+)*)\s+import\s+(.*)$")


def _relativise(src, siblings):
    out = []
    for line in src.splitlines(keepends=True):
        m = _FROM_RE.match(line.rstrip("\n"))
        if m and m.group(2) in siblings:
            line = "%sfrom .%s%s import %s\n" % (m.group(1), m.group(2), m.group(3), m.group(4))
        else:
            m = _IMPORT_RE.match(line.rstrip("\n"))
            if m:
                names = [n.strip() for n in m.group(2).split(",")]
                if any(n.split(".")[0] in siblings for n in names):
                    parts = []
                    for n in names:
                        if n.split(".")[0] in siblings:
                            parts.append("%sfrom . import %s" % (m.group(1), n))
                        else:
                            parts.append("%simport %s" % (m.group(1), n))
                    line = "\n".join(parts) + "\n"
        out.append(line)
    return "".join(out)


def convert_file(path, siblings):
    with open(path, "r", encoding="latin-1") as f:
        src = f.read()
    src = "".join(l.expandtabs(8) for l in src.splitlines(keepends=True))
    src = _convert_prints(src)
    src = _relativise(src, siblings)
    src = re.sub(r"(\w[\w\.]*)\.keys\(\)\[0\]", r"list(\1.keys())[0]", src)
    src = src.replace("idlst = dic.values()", "idlst = list(dic.values())")
    src = src.replace("string.join(time.asctime().split(':'))", "' '.join(time.asctime().split(':'))")
    src = src.replace("string.join(dat.split(' ')[1:],'_')", "'_'.join(dat.split(' ')[1:])")
    # Python 2 orders None below every number: an empty MPO-bond slice (size None) is skipped
    src = src.replace("if qops.dic[jslc].size > 0:", "if (qops.dic[jslc].size or 0) > 0:")
    base = os.path.basename(path)
    if base == "mpo_dmrg_dotutil.py":
        src = src.replace("cdimc = cdim/dim", "cdimc = cdim//dim")
    if base == "mpo_dmrg_qphys.py":
        src = src.replace("*(norb/2)", "*(norb//2)")
    # prelude after a leading docstring/comments is not needed: put at top
    return PRELUDE + src


def convert(ref):
    dst_pkg = os.path.join(OUT_ROOT, "qcmpodmrg")
    if os.path.isdir(dst_pkg):
        shutil.rmtree(dst_pkg)
    os.makedirs(dst_pkg)
    open(os.path.join(dst_pkg, "__init__.py"), "w").close()
    src_root = os.path.join(ref, "source")
    nfail = 0
    for dirpath, dirnames, filenames in os.walk(src_root):
        rel = os.path.relpath(dirpath, ref)
        out_dir = os.path.join(dst_pkg, rel)
        os.makedirs(out_dir, exist_ok=True)
        siblings = set(os.path.splitext(f)[0] for f in filenames if f.endswith(".py"))
        siblings |= set(d for d in dirnames if os.path.exists(os.path.join(dirpath, d, "__init__.py")))
        siblings.discard("__init__")
        for fn in filenames:
            if not fn.endswith(".py"):
                continue
            sp = os.path.join(dirpath, fn)
            dp = os.path.join(out_dir, fn)
            try:
                code = convert_file(sp, siblings)
                compile(code, dp, "exec")
            except Exception as e:  # keep going: only the hot-path subset must compile
                nfail += 1
                code = "raise ImportError(%r)\n" % ("py2->3 conversion failed: %s" % e)
            with open(dp, "w") as f:
                f.write(code)
        if not os.path.exists(os.path.join(out_dir, "__init__.py")):
            open(os.path.join(out_dir, "__init__.py"), "w").close()
    libs = os.path.join(dst_pkg, "libs")
    os.makedirs(libs, exist_ok=True)
    # install.sh:5-8 recipe, compiled from the source where it lies
    subprocess.check_call(["gcc", "-fPIC", "-shared", "-g", "-O2", "-o",
                           os.path.join(libs, "libqsym.so"), os.path.join(ref, "ctypes", "qsym.c")])
    return nfail


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("QCMPODMRG_REFERENCE", "/root/reference"))
    a = ap.parse_args()
    n = convert(a.ref)
    print("converted into", OUT_ROOT, "files that failed to convert:", n)
