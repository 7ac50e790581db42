"""Mechanical OKL -> C translation of the reference's LIJ kernels.

TEST INFRASTRUCTURE.  This script reads the reference's own kernel sources
where they lie (a reference checkout given on the command line) and writes
C into ``oracle/_ref/`` (git-ignored), which ``oracle/Makefile`` (target
``ref``) compiles with ``oracle/ref_driver.c`` into
``oracle/_ref/libokl_ref.so``.  Nothing of the reference is copied into the
repository: the generated files exist only in the build folder.

OKL is C with attributes.  OCCA's Serial backend turns a kernel into a
plain C function in which every ``@outer`` / ``@inner`` loop is an ordinary
loop, ``@shared`` arrays are locals, ``@barrier`` does nothing and every
``@dim`` typed variable is indexed column-major; its OpenMP backend adds
``#pragma omp parallel for`` to a kernel's outermost ``@outer`` loop.  The
rewrite below does exactly that and nothing else, so the operation order of
the translated kernels is the reference's:

* ``typedef T name @dim(d0, d1, ...);`` -> ``typedef T name;``, and inside
  every function each variable declared with such a type (parameter or
  local, pointer or array) has its calls ``v(a0, a1, ...)`` rewritten to
  ``v[(a0) + (d0)*((a1) + (d1)*(...))]`` (OCCA's ``@dim`` rule);
* ``for(init; cond; step; <attr>)`` -> ``for(init; cond; step)`` (this also
  drops the stray empty fourth clause of ``for(...; ++i;)``);
* ``@kernel``, ``@restrict``, ``@shared`` removed; ``@barrier()`` -> no-op;
* ``inline`` helpers become ``static inline``; each ``@kernel`` is exported
  as ``<file stem>__<kernel>``, because several files define kernels of the
  same name;
* ``NVAR`` and ``MAX_LINE_ELEM`` (OCCA kernel properties, ``src/main.cxx``
  ``kernelProps``) become run-time ints set by the driver, so local arrays
  sized by them are C99 variable-length arrays.

Also extracted, as C++ inside a small shim class with the reference's member
names: ``Jacobian::assembleTriBlocks`` and ``Jacobian::resizeBlockSize``
(``src/Jacobian.cxx``), the host code that packs the in-line lower blocks and
resizes the block size.

Usage: python okl2c.py --reference <checkout> --out <dir>
"""
from __future__ import annotations

import argparse
import os
import re
import sys

OKL_FILES = (
    # (path inside the checkout, stem used for exported kernel names)
    ("src/okl/lineLU_v2.okl", "lineLU_v2"),
    ("src/okl/linesmoothLU_TriBlock_v3.okl", "TriBlock_v3"),
    ("src/okl/linesmoothLU_v5.okl", "v5"),
)
JACOBIAN_CXX = "src/Jacobian.cxx"
JACOBIAN_METHODS = ("assembleTriBlocks", "resizeBlockSize")


class TranslateError(RuntimeError):
    pass


def strip_comments(src: str) -> str:
    """Removes /* */ and // comments, keeping line structure and strings."""
    out, i, n = [], 0, len(src)
    while i < n:
        c = src[i]
        if src.startswith("/*", i):
            j = src.find("*/", i + 2)
            if j < 0:
                raise TranslateError("unterminated comment")
            out.append("\n" * src.count("\n", i, j + 2))
            i = j + 2
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif c == '"':
            j = i + 1
            while j < n and src[j] != '"':
                j += 2 if src[j] == "\\" else 1
            out.append(src[i:j + 1])
            i = j + 1
        else:
            out.append(c)
            i += 1
    return "".join(out)


def match_close(s: str, i: int, open_c: str, close_c: str) -> int:
    """Index of the bracket closing the one at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == open_c:
            depth += 1
        elif s[j] == close_c:
            depth -= 1
            if depth == 0:
                return j
    raise TranslateError(f"unbalanced {open_c}{close_c} at offset {i}")


def split_top(s: str, sep: str) -> list[str]:
    """Splits s at `sep` characters outside any () [] {} nesting."""
    parts, depth, start = [], 0, 0
    for j, c in enumerate(s):
        if c in "([{":
            depth += 1
        elif c in ")]}":
            depth -= 1
        elif c == sep and depth == 0:
            parts.append(s[start:j])
            start = j + 1
    parts.append(s[start:])
    return parts


def parse_dim_typedefs(src: str) -> tuple[str, dict[str, list[str]]]:
    dims = {}

    def repl(m):
        base, name, args = m.group(1), m.group(2), m.group(3)
        dims[name] = [a.strip() for a in split_top(args, ",")]
        return f"typedef {base.strip()} {name};"

    pat = re.compile(r"typedef\s+([\w\s]+?)\s+(\w+)\s*@dim\s*\(([^)]*)\)\s*;")
    return pat.sub(repl, src), dims


def rewrite_for_loops(src: str, omp_outer: bool) -> str:
    """Drops the fourth clause of every OKL for loop.  With omp_outer, the
    first @outer/@tile loop met at each kernel's top nesting level gets
    `#pragma omp parallel for` (what OCCA's OpenMP backend emits)."""
    out, i = [], 0
    pat = re.compile(r"\bfor\s*\(")
    while True:
        m = pat.search(src, i)
        if not m:
            out.append(src[i:])
            break
        p = m.end() - 1
        q = match_close(src, p, "(", ")")
        clauses = split_top(src[p + 1:q], ";")
        if len(clauses) not in (3, 4):
            raise TranslateError(f"for loop with {len(clauses)} clauses: {src[m.start():q + 1]!r}")
        attr = clauses[3].strip() if len(clauses) == 4 else ""
        out.append(src[i:m.start()])
        if omp_outer and "@outer" in attr:  # plain @outer, or @tile(n, @outer, @inner)
            out.append("OKL_OMP_OUTER ")
        out.append("for(" + ";".join(clauses[:3]) + ")")
        i = q + 1
    return "".join(out)


def mark_first_outer_only(src: str) -> str:
    """Keeps OKL_OMP_OUTER only on the outermost @outer loop of a kernel:
    a marker inside the body of an earlier marked loop is removed."""
    out, i = [], 0
    while True:
        j = src.find("OKL_OMP_OUTER", i)
        if j < 0:
            out.append(src[i:])
            break
        out.append(src[i:j + len("OKL_OMP_OUTER")])
        # skip to the loop body and blank nested markers inside it
        k = src.find("{", j)
        if k < 0:
            raise TranslateError("@outer loop without a body")
        e = match_close(src, k, "{", "}")
        out.append(src[j + len("OKL_OMP_OUTER"):k])
        out.append(src[k:e + 1].replace("OKL_OMP_OUTER ", ""))
        i = e + 1
    return "".join(out)


def find_functions(src: str):
    """(start, name_start, name, params (open, close), body (open, close), is_kernel)
    of every top-level function definition."""
    pat = re.compile(r"(@kernel\s+)?(?:inline\s+)?void\s+(\w+)\s*\(")
    funcs, i = [], 0
    while True:
        m = pat.search(src, i)
        if not m:
            return funcs
        p = m.end() - 1
        q = match_close(src, p, "(", ")")
        k = q + 1
        while k < len(src) and src[k].isspace():
            k += 1
        if k >= len(src) or src[k] != "{":
            i = q + 1  # a declaration or a call, not a definition
            continue
        e = match_close(src, k, "{", "}")
        funcs.append((m.start(), m.start(2), m.group(2), (p, q), (k, e), bool(m.group(1))))
        i = e + 1


def index_expr(name: str, dims: list[str], args: list[str]) -> str:
    if len(args) > len(dims):
        raise TranslateError(f"{name}: {len(args)} indices for @dim{tuple(dims)}")
    expr = f"({args[-1].strip()})"
    for a, d in zip(reversed(args[:-1]), reversed(dims[:len(args) - 1])):
        expr = f"(({a.strip()}) + ({d})*{expr})"
    return f"{name}[{expr}]"


def rewrite_indexing(text: str, typed: dict[str, list[str]]) -> str:
    """Rewrites v(a, b, ...) for every @dim-typed variable v in `text`."""
    if not typed:
        return text
    pat = re.compile(r"(?<![\w.>])(" + "|".join(map(re.escape, typed)) + r")\s*\(")
    out, i = [], 0
    while True:
        m = pat.search(text, i)
        if not m:
            out.append(text[i:])
            return "".join(out)
        p = m.end() - 1
        q = match_close(text, p, "(", ")")
        args = [rewrite_indexing(a, typed) for a in split_top(text[p + 1:q], ",")]
        out.append(text[i:m.start()])
        out.append(index_expr(m.group(1), typed[m.group(1)], args))
        i = q + 1


def translate_okl(src: str, stem: str, omp: bool = True) -> tuple[str, list[str]]:
    """Returns (C source, kernel prototypes)."""
    src = strip_comments(src)
    src, dims = parse_dim_typedefs(src)
    src = rewrite_for_loops(src, omp)
    decl = re.compile(r"\b(" + "|".join(map(re.escape, dims)) + r")\s*(?:\*\s*)?(\w+)") if dims \
        else None
    pieces, protos, last = [], [], 0
    for start, name_start, name, (pp, pq), (bo, be), is_kernel in find_functions(src):
        pieces.append(src[last:start])
        head = src[start:pq + 1]
        body = src[bo:be + 1]
        typed = {}
        if decl:
            for m in decl.finditer(src[pp:be + 1]):
                typed[m.group(2)] = dims[m.group(1)]
        body = rewrite_indexing(body, typed)
        if is_kernel:
            head = head.replace("@kernel", "", 1).lstrip()
            head = re.sub(r"\bvoid\s+" + re.escape(name) + r"\s*\(", f"void {stem}__{name}(", head, 1)
            body = mark_first_outer_only(body) if omp else body
            protos.append(strip_attrs(head) + ";")
        else:
            head = re.sub(r"^\s*inline\b", "static inline", head)
            if not head.lstrip().startswith("static"):
                head = "static " + head
        pieces.append(head + "\n" + body)
        last = be + 1
    pieces.append(src[last:])
    out = strip_attrs("".join(pieces))
    if "@" in out:
        k = out.index("@")
        raise TranslateError(f"untranslated attribute near {out[k:k + 40]!r}")
    return out, protos


def strip_attrs(s: str) -> str:
    s = re.sub(r"@barrier\s*\(\s*\)", "((void)0)", s)
    s = re.sub(r"@(restrict|shared|exclusive)\b", "", s)
    return s.replace("OKL_OMP_OUTER", "OKL_OMP_OUTER_PRAGMA")


C_PRELUDE = """\
/* generated by oracle/okl2c.py from {path} -- do not edit, do not commit */
#include "okl_rt.h"
"""

RT_HEADER = """\
/* generated by oracle/okl2c.py -- do not edit, do not commit */
#ifndef OKL_RT_H
#define OKL_RT_H
extern int okl_nvar;           /* OCCA kernel property NVAR */
extern int okl_max_line_elem;  /* OCCA kernel property MAX_LINE_ELEM */
extern int okl_threads;        /* OpenMP threads of an @outer loop */
#define NVAR okl_nvar
#define MAX_LINE_ELEM okl_max_line_elem
#define p_Nblock ((NVAR + 9 - 1) / 9)
#ifdef _OPENMP
#define OKL_OMP_OUTER_PRAGMA _Pragma("omp parallel for num_threads(okl_threads)")
#else
#define OKL_OMP_OUTER_PRAGMA
#endif
#endif
"""


def extract_method(src: str, cls: str, method: str) -> str:
    m = re.search(r"\b(?:void|bool|int)\s+" + cls + r"::" + method + r"\s*\(", src)
    if not m:
        raise TranslateError(f"{cls}::{method} not found")
    p = m.end() - 1
    q = match_close(src, p, "(", ")")
    k = src.index("{", q)
    e = match_close(src, k, "{", "}")
    return src[m.start():e + 1]


CXX_SHIM = """\
/* generated by oracle/okl2c.py from {path} -- do not edit, do not commit.
 * The reference's Jacobian methods, verbatim, inside a shim of the class
 * with the members they touch (the OCCA device members left out). */
#include <cstdio>
#include <cstring>
#include <vector>

class Mesh {{
  public:
    int nvar, nelem, nintface, eftot, nline, nlineelem, max_line_nelem;
    std::vector<int> epoint, ef, fc, lines, linesize, lineface, linepoint;
}};

class Jacobian {{
  public:
    int nvar, nelem, nintface;
    std::vector<double> jacDLU, jacD, jacO1, jacO2, rhs, res, U, U0, dU, A, DinvC;
    void assembleTriBlocks(Mesh &mesh);
    void resizeBlockSize(int nvar_new);
}};

{methods}

template <class T> static std::vector<T> vec(const T *p, size_t n) {{ return std::vector<T>(p, p + n); }}

/* A packing of the reference (Jacobian.cxx assembleTriBlocks); A is
 * nv*nv*nlineelem doubles, zero where no in-line lower block exists. */
extern "C" void okl_ref_assemble_tri_blocks(int nvar, int nelem, int nintface, int nline,
        int nlineelem, const int *fc, const int *linesize, const int *linepoint,
        const int *lines, const int *lineface, const double *jacO1, const double *jacO2,
        double *A) {{
    Mesh mesh;
    mesh.nline = nline;
    int nlf = 0;
    for (int l = 0; l < nline; ++l) nlf += linesize[l];
    mesh.fc = vec(fc, 2 * (size_t)nintface);
    mesh.linesize = vec(linesize, (size_t)nline);
    mesh.linepoint = vec(linepoint, (size_t)nline + 1);
    mesh.lines = vec(lines, (size_t)nlf);
    mesh.lineface = vec(lineface, (size_t)nlf);
    Jacobian jac;
    jac.nvar = nvar; jac.nelem = nelem; jac.nintface = nintface;
    size_t bs = (size_t)nvar * nvar;
    jac.jacO1 = vec(jacO1, bs * nintface);
    jac.jacO2 = vec(jacO2, bs * nintface);
    jac.A.assign(bs * nlineelem, 0.0);
    jac.assembleTriBlocks(mesh);
    std::memcpy(A, jac.A.data(), jac.A.size() * sizeof(double));
}}

/* Jacobian.cxx resizeBlockSize on arrays read at nv_old; outputs sized for nv_new. */
extern "C" void okl_ref_resize_block_size(int nv_old, int nv_new, int nelem, int nintface,
        const double *D, const double *O1, const double *O2, const double *rhs,
        const double *U0, double *D_new, double *O1_new, double *O2_new, double *rhs_new,
        double *U0_new) {{
    Jacobian jac;
    jac.nvar = nv_old; jac.nelem = nelem; jac.nintface = nintface;
    size_t bo = (size_t)nv_old * nv_old, bn = (size_t)nv_new * nv_new;
    jac.jacD = vec(D, bo * nelem);
    jac.jacO1 = vec(O1, bo * nintface);
    jac.jacO2 = vec(O2, bo * nintface);
    jac.rhs = vec(rhs, (size_t)nv_old * nelem);
    jac.U0 = vec(U0, (size_t)nv_old * nelem);
    jac.U.assign((size_t)nv_old * nelem, 0.0);
    jac.dU.assign((size_t)nv_old * nelem, 0.0);
    jac.res.assign((size_t)nv_old * nelem, 0.0);
    jac.jacDLU.assign(bo * nelem, 0.0);
    jac.A.assign(bo * nelem, 0.0);
    jac.resizeBlockSize(nv_new);
    std::memcpy(D_new, jac.jacD.data(), bn * nelem * sizeof(double));
    std::memcpy(O1_new, jac.jacO1.data(), bn * nintface * sizeof(double));
    std::memcpy(O2_new, jac.jacO2.data(), bn * nintface * sizeof(double));
    std::memcpy(rhs_new, jac.rhs.data(), (size_t)nv_new * nelem * sizeof(double));
    std::memcpy(U0_new, jac.U0.data(), (size_t)nv_new * nelem * sizeof(double));
}}
"""


def generate(reference: str, out_dir: str) -> list[str]:
    os.makedirs(out_dir, exist_ok=True)
    written = []

    def write(name, text):
        path = os.path.join(out_dir, name)
        with open(path, "w") as f:
            f.write(text)
        written.append(path)

    write("okl_rt.h", RT_HEADER)
    protos_all, typedefs = [], {}
    for rel, stem in OKL_FILES:
        with open(os.path.join(reference, rel)) as f:
            src = f.read()
        c, protos = translate_okl(src, stem)
        write(f"okl_{stem}.c", C_PRELUDE.format(path=rel) + c)
        protos_all += protos
        for m in re.finditer(r"typedef\s+([\w\s]+?)\s+(\w+)\s*@dim", strip_comments(src)):
            typedefs[m.group(2)] = " ".join(m.group(1).split())
    hdr = ["/* generated by oracle/okl2c.py -- do not edit, do not commit */",
           "#ifndef OKL_KERNELS_H", "#define OKL_KERNELS_H", '#include "okl_rt.h"']
    hdr += [f"typedef {t} {n};" for n, t in typedefs.items()]
    hdr += [" ".join(p.split()) for p in protos_all]
    hdr += ["#endif", ""]
    write("okl_kernels.h", "\n".join(hdr))
    with open(os.path.join(reference, JACOBIAN_CXX)) as f:
        jsrc = f.read()
    methods = "\n\n".join(extract_method(jsrc, "Jacobian", m) for m in JACOBIAN_METHODS)
    write("jacobian_methods.cxx", CXX_SHIM.format(path=JACOBIAN_CXX, methods=methods))
    return written


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--reference", required=True, help="reference checkout (read only)")
    ap.add_argument("--out", required=True, help="output folder (oracle/_ref)")
    a = ap.parse_args(argv)
    for rel, _ in OKL_FILES + ((JACOBIAN_CXX, None),):
        if not os.path.exists(os.path.join(a.reference, rel)):
            print(f"okl2c: {rel} not found under {a.reference}", file=sys.stderr)
            return 2
    for p in generate(a.reference, a.out):
        print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main())
