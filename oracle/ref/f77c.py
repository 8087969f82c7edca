"""Translate the reference's fixed-form Fortran 77 kernels into C with the
same arithmetic, so that the reference's C++ (which calls them through
SAMRAI_F77_FUNC, i.e. name_ with every argument by address) can be linked
and run in an image without a Fortran compiler.

    python f77c.py file.f [file.f ...] > kernels.c

Fortran semantics kept: the type of every literal (1.0 is REAL*4, 1.d0 is
REAL*8, so `tranwt = 1.0/(1+r)` divides in single precision), mixed-mode
promotion, integer division truncating toward zero, the evaluation order
written in the source (every operation is parenthesised as parsed; compile
the output with -ffp-contract=off), DO-loop trip counts fixed at entry,
column-major arrays with declared lower bounds, and arguments by address.
Handled subset: SUBROUTINE, IMPLICIT NONE, INTEGER / REAL / DOUBLE
PRECISION / REAL*8 / LOGICAL declarations, PARAMETER, DO ... ENDDO, block
and logical IF, assignment, RETURN, CONTINUE, END, and the intrinsics
abs, dble, real, int, min, max, sign, mod, sqrt.  A routine using anything
else (complex data, CALL, GOTO, ...) is skipped and reported on stderr.

TEST INFRASTRUCTURE ONLY: part of the recipe that builds the reference into
oracle/_ref/.
"""
import re
import sys


class Unsupported(Exception):
    pass


# ---------------------------------------------------------------------------
# source form
# ---------------------------------------------------------------------------

def statements(text):
    """Logical statements (label, text in lower case) of fixed-form source:
    comment lines dropped, continuation lines joined, '!' comments cut."""
    out = []
    for raw in text.splitlines():
        if not raw.strip():
            continue
        if raw[0] in "cC*!":
            continue
        line = raw.rstrip("\n")
        label = line[:5].strip()
        cont = len(line) > 5 and line[5] not in " 0"
        body = line[6:] if len(line) > 6 else ""
        bang = body.find("!")
        if bang >= 0:
            body = body[:bang]
        body = body.lower()
        if cont:
            if not out:
                raise Unsupported("continuation without a statement")
            out[-1] = (out[-1][0], out[-1][1] + " " + body.strip())
        else:
            out.append((label, body.strip()))
    return [(lb, re.sub(r"\s+", " ", st).strip()) for lb, st in out]


# ---------------------------------------------------------------------------
# expressions
# ---------------------------------------------------------------------------

TOK = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?)
  | (?P<dot>\.(lt|le|eq|ne|gt|ge|and|or|not|true|false|eqv|neqv)\.)
  | (?P<name>[a-z_][a-z0-9_]*)
  | (?P<op>\*\*|[-+*/(),:=])
  | (?P<ws>\s+)
""", re.X)


def tokenize(s):
    toks, i = [], 0
    while i < len(s):
        m = TOK.match(s, i)
        if not m:
            raise Unsupported(f"cannot tokenize {s[i:]!r}")
        i = m.end()
        if m.lastgroup == "ws":
            continue
        toks.append((m.lastgroup, m.group(0)))
    return toks


class Node:
    def __init__(self, kind, **kw):
        self.kind = kind
        self.__dict__.update(kw)


RANK = {"i": 0, "f": 1, "d": 2}


def promote(a, b):
    if a == "l" or b == "l":
        raise Unsupported("arithmetic on logical")
    return a if RANK[a] >= RANK[b] else b


class Parser:
    def __init__(self, toks, routine):
        self.t, self.k, self.r = toks, 0, routine

    def peek(self):
        return self.t[self.k] if self.k < len(self.t) else (None, None)

    def take(self, val=None):
        tk = self.peek()
        if val is not None and tk[1] != val:
            raise Unsupported(f"expected {val!r}, got {tk[1]!r}")
        self.k += 1
        return tk

    def done(self):
        return self.k >= len(self.t)

    # precedence climbing over the Fortran levels
    def expr(self):
        return self.or_()

    def or_(self):
        a = self.and_()
        while self.peek()[1] == ".or.":
            self.take()
            a = Node("bin", op="||", a=a, b=self.and_(), ty="l")
        return a

    def and_(self):
        a = self.not_()
        while self.peek()[1] == ".and.":
            self.take()
            a = Node("bin", op="&&", a=a, b=self.not_(), ty="l")
        return a

    def not_(self):
        if self.peek()[1] == ".not.":
            self.take()
            return Node("un", op="!", a=self.not_(), ty="l")
        return self.rel()

    RELOPS = {".lt.": "<", ".le.": "<=", ".eq.": "==", ".ne.": "!=", ".gt.": ">", ".ge.": ">="}

    def rel(self):
        a = self.add()
        op = self.peek()[1]
        if op in self.RELOPS:
            self.take()
            b = self.add()
            promote(a.ty, b.ty)
            return Node("bin", op=self.RELOPS[op], a=a, b=b, ty="l")
        return a

    def add(self):
        # a leading sign applies to the first term (Fortran level 2)
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            t = self.mul()
            a = Node("un", op=op, a=t, ty=t.ty)
        else:
            a = self.mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            b = self.mul()
            a = Node("bin", op=op, a=a, b=b, ty=promote(a.ty, b.ty))
        return a

    def mul(self):
        a = self.pow_()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            b = self.pow_()
            a = Node("bin", op=op, a=a, b=b, ty=promote(a.ty, b.ty))
        return a

    def pow_(self):
        a = self.prim()
        if self.peek()[1] == "**":
            raise Unsupported("exponentiation")
        return a

    def prim(self):
        kind, val = self.take()
        if kind == "num":
            if "d" in val:
                return Node("num", text=val.replace("d", "e"), ty="d")
            if "." in val or "e" in val:
                return Node("num", text=val, ty="f")
            return Node("num", text=val, ty="i")
        if kind == "dot" and val in (".true.", ".false."):
            return Node("num", text="1" if val == ".true." else "0", ty="l")
        if val == "(":
            e = self.expr()
            self.take(")")
            return Node("paren", a=e, ty=e.ty)
        if kind == "name":
            if self.peek()[1] == "(":
                self.take("(")
                args = []
                if self.peek()[1] != ")":
                    args.append(self.expr())
                    while self.peek()[1] == ",":
                        self.take()
                        args.append(self.expr())
                self.take(")")
                return self.r.ref(val, args)
            return self.r.scalar(val)
        raise Unsupported(f"unexpected token {val!r}")


CT = {"i": "int", "f": "float", "d": "double", "l": "int"}


def emit(n):
    """C text of an expression node, parenthesised as parsed."""
    k = n.kind
    if k == "num":
        if n.ty == "f":
            t = n.text
            if "." not in t and "e" not in t:
                t += "."
            return f"{t}f"
        if n.ty == "d":
            return f"{n.text}" if ("." in n.text or "e" in n.text) else f"{n.text}.0"
        return n.text
    if k == "paren":
        return f"({emit(n.a)})"
    if k == "un":
        return f"({n.op}{emit(n.a)})"
    if k == "bin":
        return f"({emit(n.a)} {n.op} {emit(n.b)})"
    if k == "var":
        return n.text
    if k == "call":
        return n.text
    raise Unsupported(k)


# ---------------------------------------------------------------------------
# routines
# ---------------------------------------------------------------------------

TYPES = [("double precision", "d"), ("real*8", "d"), ("real*4", "f"), ("real", "f"),
         ("integer", "i"), ("logical", "l")]


def split_top(s, sep=","):
    """Split at `sep` outside parentheses."""
    out, depth, cur = [], 0, []
    for c in s:
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c == sep and depth == 0:
            out.append("".join(cur).strip())
            cur = []
        else:
            cur.append(c)
    if cur or out:
        out.append("".join(cur).strip())
    return out


def match_paren(s, i):
    """Index of the ')' closing the '(' at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise Unsupported("unbalanced parentheses")


class Routine:
    def __init__(self, name, args):
        self.name, self.args = name, args
        self.types = {}      # name -> i/f/d/l
        self.dims = {}       # name -> [(lo, hi)] as Fortran expression text
        self.params = {}     # name -> expression text
        self.implicit_none = False
        self.body = []       # C lines
        self.indent = 1

    # -- symbols
    def type_of(self, n):
        if n in self.types:
            return self.types[n]
        if self.implicit_none:
            raise Unsupported(f"undeclared {n}")
        return "i" if n[0] in "ijklmn" else "f"

    def cname(self, n):
        return f"f_{n}"

    def scalar(self, n):
        ty = self.type_of(n)
        if n in self.dims:
            raise Unsupported(f"whole array {n} in an expression")
        if n in self.args:
            return Node("var", text=f"(*{self.cname(n)})", ty=ty)
        return Node("var", text=self.cname(n), ty=ty)

    def ref(self, n, args):
        if n in self.dims:
            if len(args) != len(self.dims[n]):
                raise Unsupported(f"rank of {n}")
            terms = []
            for a, d in enumerate(range(len(args))):
                terms.append(f"(long)({emit(args[a])} - {self.cname(n)}_lo{a})")
            idx = terms[-1]
            for a in range(len(args) - 2, -1, -1):
                idx = f"{terms[a]} + {self.cname(n)}_ext{a} * ({idx})"
            return Node("var", text=f"{self.cname(n)}[{idx}]", ty=self.type_of(n))
        return self.intrinsic(n, args)

    def intrinsic(self, n, args):
        tys = [a.ty for a in args]
        cs = [emit(a) for a in args]
        if n in ("abs", "dabs", "iabs"):
            ty = tys[0]
            f = {"d": "fabs", "f": "fabsf", "i": "abs"}[ty]
            return Node("call", text=f"{f}({cs[0]})", ty=ty)
        if n in ("dble", "dfloat"):
            return Node("call", text=f"((double)({cs[0]}))", ty="d")
        if n in ("real", "float", "sngl"):
            return Node("call", text=f"((float)({cs[0]}))", ty="f")
        if n == "int":
            return Node("call", text=f"((int)({cs[0]}))", ty="i")
        if n in ("min", "max", "min0", "max0", "dmin1", "dmax1", "amin1", "amax1"):
            ty = tys[0]
            for t in tys[1:]:
                if t != ty:
                    raise Unsupported(f"mixed-type {n}")
            base = "min" if "min" in n else "max"
            text = cs[0]
            for c in cs[1:]:
                text = f"f77_{base}_{ty}({text}, {c})"
            return Node("call", text=text, ty=ty)
        if n in ("sign", "dsign", "isign"):
            ty = promote(tys[0], tys[1])
            if tys[0] != tys[1]:
                raise Unsupported("mixed-type sign")
            return Node("call", text=f"f77_sign_{ty}({cs[0]}, {cs[1]})", ty=ty)
        if n == "mod":
            if tys != ["i", "i"]:
                raise Unsupported("non-integer mod")
            return Node("call", text=f"({cs[0]} % {cs[1]})", ty="i")
        if n in ("sqrt", "dsqrt"):
            f = "sqrt" if tys[0] == "d" else "sqrtf"
            return Node("call", text=f"{f}({cs[0]})", ty=tys[0])
        raise Unsupported(f"function {n}")

    def expr(self, text):
        p = Parser(tokenize(text), self)
        e = p.expr()
        if not p.done():
            raise Unsupported(f"trailing tokens in {text!r}")
        return e

    def line(self, s):
        self.body.append("   " * self.indent + s)

    # -- declarations
    def declare(self, ty, rest):
        for item in split_top(rest):
            m = re.match(r"([a-z_][a-z0-9_]*)\s*(\((.*)\))?$", item)
            if not m:
                raise Unsupported(f"declaration {item!r}")
            n = m.group(1)
            self.types[n] = ty
            if m.group(3) is not None:
                dims = []
                for d in split_top(m.group(3)):
                    lo, sep, hi = d.partition(":")
                    dims.append(("1", lo) if not sep else (lo, hi))
                self.dims[n] = dims


def assign_target(st):
    """Split `lhs = rhs` at the top-level '=' (None if not an assignment)."""
    depth = 0
    for i, c in enumerate(st):
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        elif c == "=" and depth == 0:
            return st[:i].strip(), st[i + 1:].strip()
    return None


def translate_routine(r, stmts):
    """C source of one routine; stmts are its statements after the header."""
    decl_done = False
    pre = []   # parameter and extent set-up, emitted after locals
    open_blocks = []
    i = 0
    while i < len(stmts):
        label, st = stmts[i]
        i += 1
        if label:
            raise Unsupported("statement labels")
        if not decl_done:
            if st == "implicit none":
                r.implicit_none = True
                continue
            matched = False
            for kw, ty in TYPES:
                if st.startswith(kw + " ") or st == kw:
                    r.declare(ty, st[len(kw):].strip())
                    matched = True
                    break
            if matched:
                continue
            m = re.match(r"parameter\s*\((.*)\)$", st)
            if m:
                for item in split_top(m.group(1)):
                    n, _, v = item.partition("=")
                    r.params[n.strip()] = v.strip()
                continue
            if st.startswith(("double complex", "complex", "character", "common", "data ",
                              "save", "equivalence", "external", "intrinsic", "include")):
                raise Unsupported(st.split()[0])
            decl_done = True
            emit_prologue(r, pre)
        # executable statements
        if st in ("end",):
            break
        if st == "return":
            r.line("return;")
            continue
        if st == "continue":
            r.line(";")
            continue
        if st in ("enddo", "end do"):
            if not open_blocks or open_blocks.pop() != "do":
                raise Unsupported("unmatched enddo")
            r.indent -= 1
            r.line("}")
            r.indent -= 1
            r.line("}")
            continue
        if st in ("endif", "end if"):
            if not open_blocks or open_blocks.pop() != "if":
                raise Unsupported("unmatched endif")
            r.indent -= 1
            r.line("}")
            continue
        if st == "else":
            r.indent -= 1
            r.line("} else {")
            r.indent += 1
            continue
        m = re.match(r"else ?if\s*\(", st)
        if m:
            j = match_paren(st, st.index("("))
            if st[j + 1:].strip() != "then":
                raise Unsupported(st)
            c = r.expr(st[st.index("(") + 1:j])
            r.indent -= 1
            r.line(f"}} else if ({emit(c)}) {{")
            r.indent += 1
            continue
        m = re.match(r"do\s+([a-z_][a-z0-9_]*)\s*=(.*)$", st)
        if m:
            v = m.group(1)
            parts = split_top(m.group(2))
            if len(parts) not in (2, 3):
                raise Unsupported(st)
            lo, hi = r.expr(parts[0]), r.expr(parts[1])
            stp = r.expr(parts[2]) if len(parts) == 3 else None
            if r.type_of(v) != "i":
                raise Unsupported("non-integer DO variable")
            var = emit(r.scalar(v))
            sc = emit(stp) if stp is not None else "1"
            # trip count fixed at entry: max(0, (hi - lo + step) / step)
            r.line("{")
            r.indent += 1
            r.line(f"const int f77_step = {sc};")
            r.line(f"int f77_trip = ({emit(hi)} - ({emit(lo)}) + f77_step) / f77_step;")
            r.line(f"for ({var} = {emit(lo)}; f77_trip > 0; --f77_trip, {var} += f77_step) {{")
            r.indent += 1
            open_blocks.append("do")
            continue
        if st.startswith("if") and st[2:].lstrip().startswith("("):
            k = st.index("(")
            j = match_paren(st, k)
            c = r.expr(st[k + 1:j])
            rest = st[j + 1:].strip()
            if rest == "then":
                r.line(f"if ({emit(c)}) {{")
                r.indent += 1
                open_blocks.append("if")
            else:
                r.line(f"if ({emit(c)}) {{")
                r.indent += 1
                translate_simple(r, rest)
                r.indent -= 1
                r.line("}")
            continue
        translate_simple(r, st)
    if open_blocks:
        raise Unsupported("unterminated block")
    return assemble(r, pre)


def translate_simple(r, st):
    if st == "return":
        r.line("return;")
        return
    if st == "continue":
        r.line(";")
        return
    a = assign_target(st)
    if a is None:
        raise Unsupported(f"statement {st!r}")
    lhs, rhs = a
    lt = r.expr(lhs)
    if lt.kind != "var":
        raise Unsupported(f"assignment to {lhs!r}")
    rt = r.expr(rhs)
    r.line(f"{lt.text} = {emit(rt)};")


def emit_prologue(r, pre):
    """Parameters, locals and array extents (evaluated at entry)."""
    for n, v in r.params.items():
        ty = r.type_of(n)
        pre.append(f"const {CT[ty]} {r.cname(n)} = ({CT[ty]})({emit(r.expr(v))});")
    for n, ty in r.types.items():
        if n in r.args or n in r.params:
            continue
        if n in r.dims:
            continue
        pre.append(f"{CT[ty]} {r.cname(n)};")
    for n, dims in r.dims.items():
        for a, (lo, hi) in enumerate(dims):
            pre.append(f"const long {r.cname(n)}_lo{a} = {emit(r.expr(lo))};")
            if hi.strip() != "*":
                pre.append(f"const long {r.cname(n)}_ext{a} = "
                           f"{emit(r.expr(hi))} - {r.cname(n)}_lo{a} + 1;")
        if n not in r.args:
            size = " * ".join(f"{r.cname(n)}_ext{a}" for a in range(len(dims)))
            pre.append(f"{CT[r.type_of(n)]} {r.cname(n)}[{size}];")
    for n in r.types:
        pre.append(f"(void){r.cname(n)};")


def assemble(r, pre):
    params = []
    for a in r.args:
        ty = r.type_of(a)
        params.append(f"{CT[ty]} *{r.cname(a)}")
    out = [f"void {r.name}_({', '.join(params) if params else 'void'})", "{"]
    out += ["   " + p for p in pre]
    out += r.body
    out.append("}")
    return "\n".join(out)


PRELUDE = """/* Generated by oracle/ref/f77c.py from the reference's Fortran kernels. */
#include <math.h>
#include <stdlib.h>
static inline int f77_min_i(int a, int b) { return a < b ? a : b; }
static inline int f77_max_i(int a, int b) { return a > b ? a : b; }
static inline float f77_min_f(float a, float b) { return a < b ? a : b; }
static inline float f77_max_f(float a, float b) { return a > b ? a : b; }
static inline double f77_min_d(double a, double b) { return a < b ? a : b; }
static inline double f77_max_d(double a, double b) { return a > b ? a : b; }
static inline int f77_sign_i(int a, int b) { int m = a < 0 ? -a : a; return b >= 0 ? m : -m; }
static inline float f77_sign_f(float a, float b) { return copysignf(fabsf(a), b); }
static inline double f77_sign_d(double a, double b) { return copysign(fabs(a), b); }
"""


def translate(text, only=None, log=sys.stderr):
    """C source of every supported routine in `text` (or those in `only`)."""
    stmts = statements(text)
    out, names = [], []
    i = 0
    while i < len(stmts):
        label, st = stmts[i]
        m = re.match(r"subroutine\s+([a-z_][a-z0-9_]*)\s*\((.*)\)$", st)
        if not m:
            i += 1
            continue
        name = m.group(1)
        args = [a.strip() for a in m.group(2).split(",") if a.strip()]
        j = i + 1
        while j < len(stmts) and stmts[j][1] != "end":
            j += 1
        body = stmts[i + 1:j + 1]
        i = j + 1
        if only is not None and name not in only:
            continue
        r = Routine(name, args)
        try:
            out.append(translate_routine(r, body))
            names.append(name)
        except Unsupported as e:
            print(f"f77c: skipped {name}: {e}", file=log)
    return out, names


def main(argv):
    chunks, allnames = [PRELUDE], []
    for f in argv:
        with open(f) as fh:
            c, names = translate(fh.read())
        chunks += c
        allnames += names
    sys.stdout.write("\n\n".join(chunks) + "\n")
    print(f"f77c: {len(allnames)} routines", file=sys.stderr)


if __name__ == "__main__":
    main(sys.argv[1:])
