"""A translator of the Fortran 90 subset the reference's solver modules use into Python/numpy.

TEST INFRASTRUCTURE ONLY (golden-vector generation): it reads the reference's own
``derivs.F90``, ``nseq.F90`` and ``timeIntegration.F90`` unmodified and turns each subroutine
into a Python function over numpy arrays, so that the reference's arithmetic can be run in
a container without a Fortran compiler.  The generator script beside it runs those
functions on small cases and stores inputs and outputs as fixtures; the oracle is then
checked against the fixtures by the CPU tests.  Nothing of the reference is copied into the
repository: the source is read at generation time.

Covered: subroutines with explicit-shape, automatic and assumed-shape array dummies (any
lower bounds), real*8 / integer declarations, whole-array and array-section assignments
(evaluated element by element with numpy, the same IEEE operations in the same order as
the Fortran expression tree), do loops with steps, if / else if / else blocks, one-line ifs,
select case, call, array constructors, SAVE variables (with initialisers) and allocatable
arrays with allocate, and the intrinsics modulo, mod, sqrt / dsqrt, abs, max, min, dble,
sum (added in array-element order), atan / datan, sin / dsin.  Array sections passed to a
subroutine are numpy views, so intent(inout) dummies write through; MPI reductions on one
rank copy their input to their output.  ``include`` lines are spliced in from texts the
caller supplies (the generated disturbance and forcing hooks, written by the repository's
emitter the way the reference's generator writes them) or dropped.  Default-real literals
and variables are single precision, as in Fortran.  Not covered (absent from these files):
strings, pointers, complex numbers, where / forall.
"""
from __future__ import annotations

import keyword
import re

import numpy as _np

# ---- source preprocessing ----------------------------------------------------------------


def _strip_comment(line):
    out, q = [], None
    for ch in line:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        elif ch == "!":
            break
        else:
            out.append(ch)
    return "".join(out)


def logical_lines(text):
    """Comment-free, continuation-joined, lower-cased statements."""
    lines, buf = [], ""
    for raw in text.replace("\t", "    ").splitlines():
        s = _strip_comment(raw).rstrip()
        if not s.strip():
            continue
        t = s.strip()
        if buf:
            if t.startswith("&"):
                t = t[1:]
            buf += " " + t.strip()
        else:
            buf = t
        if buf.endswith("&"):
            buf = buf[:-1].rstrip()
            continue
        lines.append(buf.lower())
        buf = ""
    if buf:
        lines.append(buf.lower())
    return lines


# ---- expressions -------------------------------------------------------------------------

_TOK = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?)
  | (?P<dot>\.(eq|ne|lt|le|gt|ge|and|or|not|true|false|eqv|neqv)\.)
  | (?P<name>[a-z_][a-z0-9_]*)
  | (?P<op>\(/|/\)|\*\*|==|/=|<=|>=|<|>|\*|/|\+|-|\(|\)|,|:)
  | (?P<ws>\s+)
""", re.X)


def tokenize(s):
    toks, i = [], 0
    while i < len(s):
        m = _TOK.match(s, i)
        if not m:
            raise SyntaxError(f"cannot tokenize {s[i:]!r} in {s!r}")
        i = m.end()
        k = m.lastgroup
        if k == "ws":
            continue
        v = m.group(k)
        if k == "num":
            # kind: 0 integer, 4 default real (single precision), 8 double (d exponent)
            kind = 8 if "d" in v else (4 if ("." in v or "e" in v) else 0)
            toks.append(("num", v.replace("d", "e"), kind))
        elif k == "dot":
            toks.append(("op", v, None))
        else:
            toks.append((k, v, None))
    toks.append(("end", None, None))
    return toks


class Node:
    __slots__ = ("kind", "a", "b", "c")

    def __init__(self, kind, a=None, b=None, c=None):
        self.kind, self.a, self.b, self.c = kind, a, b, c


_BIN = {  # Fortran precedence, low to high
    ".eqv.": 1, ".neqv.": 1, ".or.": 2, ".and.": 3,
    "==": 5, "/=": 5, "<": 5, "<=": 5, ">": 5, ">=": 5,
    ".eq.": 5, ".ne.": 5, ".lt.": 5, ".le.": 5, ".gt.": 5, ".ge.": 5,
    "+": 6, "-": 6, "*": 7, "/": 7, "**": 9,
}


class Parser:
    def __init__(self, s):
        self.t = tokenize(s)
        self.i = 0

    def peek(self):
        return self.t[self.i]

    def take(self, v=None):
        tok = self.t[self.i]
        if v is not None and tok[1] != v:
            raise SyntaxError(f"expected {v!r}, got {tok[1]!r}")
        self.i += 1
        return tok

    def expr(self, minp=0):
        tok = self.peek()
        if tok[1] == ".not.":
            self.take()
            left = Node("not", self.expr(4))
        elif tok[1] in ("-", "+") and tok[0] == "op":
            self.take()
            # Fortran: unary minus/plus binds like binary +/- (below * and /)
            left = Node("neg" if tok[1] == "-" else "pos", self.expr(7))
        else:
            left = self.atom()
        while True:
            tok = self.peek()
            op = tok[1]
            if tok[0] != "op" or op not in _BIN:
                break
            p = _BIN[op]
            if p < minp:
                break
            self.take()
            right = self.expr(p if op == "**" else p + 1)
            left = Node("bin", op, left, right)
        return left

    def atom(self):
        tok = self.take()
        if tok[0] == "num":
            return Node("num", tok[1], tok[2])
        if tok[1] in (".true.", ".false."):
            return Node("bool", tok[1] == ".true.")
        if tok[1] == "(":
            e = self.expr()
            self.take(")")
            return Node("paren", e)
        if tok[1] == "(/":  # array constructor
            items = [self.expr()]
            while self.peek()[1] == ",":
                self.take()
                items.append(self.expr())
            self.take("/)")
            return Node("arr", items)
        if tok[0] == "name":
            if self.peek()[1] == "(":
                self.take("(")
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.subscript())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return Node("ref", tok[1], args)
            return Node("name", tok[1])
        raise SyntaxError(f"unexpected token {tok}")

    def subscript(self):
        lo = hi = None
        if self.peek()[1] != ":":
            lo = self.expr()
            if self.peek()[1] != ":":
                return lo
        self.take(":")
        if self.peek()[1] not in (",", ")"):
            hi = self.expr()
        return Node("slice", lo, hi)


def parse_expr(s):
    p = Parser(s)
    e = p.expr()
    if p.peek()[0] != "end":
        raise SyntaxError(f"trailing input in {s!r}")
    return e


# ---- runtime helpers of the generated code -------------------------------------------------

def _div(a, b):
    """Fortran division: integer operands truncate toward zero, anything else divides."""
    if isinstance(a, (int, _np.integer)) and isinstance(b, (int, _np.integer)):
        q = abs(int(a)) // abs(int(b))
        return q if (a >= 0) == (b >= 0) else -q
    return a / b


def _modulo(a, b):
    return a % b  # Fortran modulo takes the sign of b, as Python's % does


def _mod(a, b):
    return a - int(_div(a, b)) * b if isinstance(a, (int, _np.integer)) else _np.fmod(a, b)


def _max(*a):
    r = a[0]
    for x in a[1:]:
        r = _np.maximum(r, x)
    return r


def _min(*a):
    r = a[0]
    for x in a[1:]:
        r = _np.minimum(r, x)
    return r


def _sum(a):
    """Fortran sum: the elements added one after the other in array-element (column-major)
    order, as a sequential loop does (numpy's own reduction adds pairwise)."""
    a = _np.asarray(a)
    return _np.cumsum(_np.ravel(a, order="F"))[-1] if a.size else 0.0


def _r4(v):
    """A value stored in a default-real (single-precision) variable."""
    return float(_np.float32(v)) if _np.ndim(v) == 0 else _np.asarray(v, dtype=_np.float32).astype(_np.float64)


def _frange(a, b, s=1):
    return range(int(a), int(b) + (1 if s > 0 else -1), int(s))


_INTRINSIC = {
    "modulo": "_modulo", "mod": "_mod", "sqrt": "_np.sqrt", "dsqrt": "_np.sqrt", "abs": "_np.abs",
    "dabs": "_np.abs", "max": "_max", "min": "_min", "dble": "_np.float64", "exp": "_np.exp",
    "dexp": "_np.exp", "tanh": "_np.tanh", "sin": "_np.sin", "cos": "_np.cos", "sum": "_sum",
    "dsin": "_np.sin", "dcos": "_np.cos", "datan": "_np.arctan", "atan": "_np.arctan",
}

# subroutines whose second argument receives the first (MPI reductions on one rank): their
# results are scalars, which a Python call could not write back
_COPY_OUT = ("mpi_allreduce", "mpi_reduce")


def _pyname(n):
    return n + "_" if keyword.iskeyword(n) or n in ("print", "range", "len") else n


# ---- translation -----------------------------------------------------------------------------

class Scope:
    def __init__(self, globals_arrays):
        self.arrays = dict(globals_arrays)  # name -> list of lower-bound code strings
        self.ints = set()
        self.r4 = set()                     # default-real (single precision) variables
        self.saved = {}                     # SAVE variable -> its module-level Python name

    def lb(self, name, k):
        return self.arrays[name][k]


def emit(e, sc):
    k = e.kind
    if k == "num":
        if e.b == 8:
            return repr(float(e.a))
        if e.b == 4:  # a default-real literal is single precision, widened where it meets real*8
            return repr(float(_np.float32(e.a)))
        return str(int(e.a))
    if k == "arr":
        return "_np.array([" + ", ".join(emit(x, sc) for x in e.a) + "], dtype=_np.float64)"
    if k == "bool":
        return "True" if e.a else "False"
    if k == "name":
        return sc.saved.get(e.a, _pyname(e.a))
    if k == "paren":
        return "(" + emit(e.a, sc) + ")"
    if k == "neg":
        return "(-" + emit(e.a, sc) + ")"
    if k == "pos":
        return emit(e.a, sc)
    if k == "not":
        return "(not " + emit(e.a, sc) + ")"
    if k == "bin":
        op, l, r = e.a, emit(e.b, sc), emit(e.c, sc)
        if op == "/":
            return f"_div({l}, {r})"
        if op == "**":
            return f"({l} ** {r})"
        py = {".eq.": "==", ".ne.": "!=", "/=": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">=",
              ".and.": "and", ".or.": "or", ".eqv.": "==", ".neqv.": "!="}.get(op, op)
        return f"({l} {py} {r})"
    if k == "ref":
        name, args = e.a, e.b
        if name in sc.arrays:
            subs = []
            for j, s in enumerate(args):
                lb = sc.lb(name, j)
                off = "" if lb == "1" else f"({lb})"
                if s.kind == "slice":
                    lo = "" if s.a is None else (f"({emit(s.a, sc)})-1" if not off else f"({emit(s.a, sc)})-{off}")
                    hi = "" if s.b is None else (f"({emit(s.b, sc)})" if not off else f"({emit(s.b, sc)})-{off}+1")
                    subs.append(f"{lo}:{hi}")
                else:
                    subs.append(f"({emit(s, sc)})-1" if not off else f"({emit(s, sc)})-{off}")
            return f"{sc.saved.get(name, _pyname(name))}[{', '.join(subs)}]"
        fn = _INTRINSIC.get(name, _pyname(name))
        return f"{fn}({', '.join(emit(s, sc) for s in args)})"
    raise ValueError(k)


def _split_top(s, sep=","):
    out, depth, cur = [], 0, []
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [x.strip() for x in out]


def _close_paren(s, i):
    """Index of the parenthesis closing the one at s[i]."""
    depth = 0
    for j in range(i, len(s)):
        if s[j] == "(":
            depth += 1
        elif s[j] == ")":
            depth -= 1
            if depth == 0:
                return j
    raise SyntaxError(f"unbalanced parentheses in {s!r}")


def _assign_split(s):
    """Position of the assignment '=' of a statement, or -1."""
    depth = 0
    for i, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            if s[i + 1:i + 2] == "=" or s[i - 1:i] in ("=", "/", "<", ">"):
                continue
            return i
    return -1


_DECL = re.compile(r"^(real\s*\*\s*8|real|integer|double\s+precision|logical)\b")
SAVED_INIT = {}    # module-level name of a SAVE variable -> its initialiser (Fortran text) or None
ALLOC_DTYPE = {}   # (subroutine, allocatable array) -> numpy dtype of its allocation


def _parse_dims(spec):
    """'(a:b, :, n)' contents -> list of (lo, hi) expression strings, ('', '') for ':'."""
    dims = []
    for d in _split_top(spec):
        if d == ":":
            dims.append(("", ""))
        else:
            parts = _split_top(d, ":")
            dims.append((parts[0], parts[1]) if len(parts) == 2 else ("1", parts[0]))
    return dims


class Subroutine:
    def __init__(self, name, args, body):
        self.name, self.args, self.body = name, args, body


def split_subroutines(lines, include_texts=None):
    subs, cur, includes = [], None, []
    expanded = []
    for s in lines:
        m = re.match(r"^include\s+'([^']*)'$", s)
        if m and include_texts and m.group(1) in include_texts:
            expanded += logical_lines(include_texts[m.group(1)])
        else:
            expanded.append(s)
    for s in expanded:
        m = re.match(r"^subroutine\s+([a-z_][a-z0-9_]*)\s*(\((.*)\))?\s*$", s)
        if m:
            args = [a.strip() for a in (m.group(3) or "").split(",") if a.strip()]
            cur = Subroutine(m.group(1), args, [])
            continue
        if re.match(r"^end\s*subroutine\b", s):
            subs.append(cur)
            cur = None
            continue
        if cur is None:
            continue  # module, use, contains, end module
        if s.startswith("include "):
            includes.append(s)
            continue
        cur.body.append(s)
    return subs, includes


def translate_subroutine(sub, globals_arrays, trace=None):
    sc = Scope(globals_arrays)
    # dummy names: duplicates (a list that names one argument twice) get placeholders
    seen, params = set(), []
    for a in sub.args:
        if a in seen:
            params.append(f"{_pyname(a)}__dup{len(params)}")
        else:
            seen.add(a)
            params.append(_pyname(a))
    out = [f"def {_pyname(sub.name)}({', '.join(params)}):"]
    ind = 1
    pro = []
    stack = []  # open constructs: 'do', 'if', ('select', var)
    nsel = 0

    def w(line):
        out.append("    " * ind + line)

    body = []
    for s in sub.body:
        if s in ("implicit none",) or s.startswith("use "):
            continue
        md = _DECL.match(s)
        if md and ("::" in s or s[md.end():].lstrip().startswith(",")):
            typ = md.group(1)
            attrs, _, ents = s.partition("::")
            dims = None
            alist = _split_top(attrs)[1:]
            save = "save" in alist
            alloc = "allocatable" in alist
            for at in alist:
                if at.startswith("dimension"):
                    dims = _parse_dims(at[at.index("(") + 1:_close_paren(at, at.index("("))])
            for ent in _split_top(ents):
                init = None
                if "=" in ent and "(" not in ent.split("=")[0]:
                    ent, init = (x.strip() for x in ent.split("=", 1))
                nm, edims = ent, dims
                if "(" in ent:
                    nm = ent[:ent.index("(")].strip()
                    edims = _parse_dims(ent[ent.index("(") + 1:_close_paren(ent, ent.index("("))])
                if typ.startswith("integer"):
                    sc.ints.add(nm)
                if typ == "real":
                    sc.r4.add(nm)
                if save or init is not None:  # SAVE (an initialiser implies it): module-level state
                    gname = "_sv_%s_%s" % (sub.name, nm)
                    sc.saved[nm] = gname
                    SAVED_INIT[gname] = None if init is None else init
                if edims is None:
                    continue
                lbs = []
                for lo, hi in edims:
                    lbs.append("1" if lo in ("", "1") else emit(parse_expr(lo), sc))
                sc.arrays[nm] = lbs
                if alloc:
                    ALLOC_DTYPE[(sub.name, nm)] = "_np.int64" if typ.startswith("integer") else "_np.float64"
                    continue
                if nm not in sub.args:  # automatic local array
                    shape = ", ".join(f"({emit(parse_expr(hi), sc)})-({emit(parse_expr(lo), sc)})+1"
                                      for lo, hi in edims)
                    dt = "_np.int64" if typ.startswith("integer") else "_np.float64"
                    pro.append(f"{_pyname(nm)} = _np.zeros(({shape},), dtype={dt})")
            continue
        body.append(s)
    if sc.saved:
        w("global " + ", ".join(sorted(sc.saved.values())))
    for p in pro:
        w(p)
    if trace is not None:
        w(f"_trace.append({sub.name!r})")

    def stmt(s):
        nonlocal ind, nsel
        if s.startswith("call "):
            rest = s[5:].strip()
            if "(" in rest:
                nm = rest[:rest.index("(")].strip()
                args = _split_top(rest[rest.index("(") + 1:_close_paren(rest, rest.index("("))])
                if nm in _COPY_OUT:
                    w(f"{emit(parse_expr(args[1]), sc)} = {emit(parse_expr(args[0]), sc)}")
                    return
                w(f"{_pyname(nm)}({', '.join(emit(parse_expr(a), sc) for a in args)})")
            else:
                w(f"{_pyname(rest)}()")
            return
        if s == "return":
            w("return")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", s)
        if m:
            for ent in _split_top(m.group(1)):
                nm = ent[:ent.index("(")].strip()
                dims = _split_top(ent[ent.index("(") + 1:_close_paren(ent, ent.index("("))])
                shape = ", ".join(emit(parse_expr(d), sc) for d in dims)
                dt = ALLOC_DTYPE.get((sub.name, nm), "_np.float64")
                w(f"{sc.saved.get(nm, _pyname(nm))} = _np.zeros(({shape},), dtype={dt})")
            return
        if s.startswith("deallocate"):
            return
        if s == "cycle":
            w("continue")
            return
        if s == "exit":
            w("break")
            return
        k = _assign_split(s)
        if k < 0:
            raise SyntaxError(f"unsupported statement in {sub.name}: {s!r}")
        lhs, rhs = s[:k].strip(), s[k + 1:].strip()
        r = emit(parse_expr(rhs), sc)
        le = parse_expr(lhs)
        if le.kind == "name" and le.a in sc.arrays:
            w(f"{sc.saved.get(le.a, _pyname(le.a))}[...] = {r}")
        elif le.kind == "name" and le.a in sc.r4:
            w(f"{emit(le, sc)} = _r4({r})")
        else:
            w(f"{emit(le, sc)} = {r}")

    for s in body:
        m = re.match(r"^do\s+([a-z_][a-z0-9_]*)\s*=\s*(.*)$", s)
        if m:
            lim = _split_top(m.group(2))
            args = ", ".join(emit(parse_expr(x), sc) for x in lim)
            w(f"for {_pyname(m.group(1))} in _frange({args}):")
            ind += 1
            w("pass")
            stack.append("do")
            continue
        if re.match(r"^end\s*do$", s):
            assert stack.pop() == "do", (sub.name, s)
            ind -= 1
            continue
        m = re.match(r"^(else\s*)?if\s*\(", s)
        if m:
            i0 = s.index("(")
            j = _close_paren(s, i0)
            cond = emit(parse_expr(s[i0 + 1:j]), sc)
            tail = s[j + 1:].strip()
            if m.group(1):
                ind -= 1
                w(f"elif {cond}:")
                ind += 1
                w("pass")
            elif tail == "then":
                w(f"if {cond}:")
                ind += 1
                w("pass")
                stack.append("if")
            else:
                w(f"if {cond}:")
                ind += 1
                stmt(tail)
                ind -= 1
            continue
        if s == "else":
            ind -= 1
            w("else:")
            ind += 1
            w("pass")
            continue
        if re.match(r"^end\s*if$", s):
            assert stack.pop() == "if", (sub.name, s)
            ind -= 1
            continue
        m = re.match(r"^select\s*case\s*\((.*)\)$", s)
        if m:
            nsel += 1
            var = f"_sel{nsel}"
            w(f"{var} = {emit(parse_expr(m.group(1)), sc)}")
            stack.append(("select", var, [False]))
            continue
        m = re.match(r"^case\s*(\((.*)\)|default)$", s)
        if m:
            top = stack[-1]
            assert top[0] == "select", (sub.name, s)
            if top[2][0]:
                ind -= 1
            if m.group(1) == "default":
                w("else:" if top[2][0] else "if True:")
            else:
                vals = ", ".join(emit(parse_expr(v), sc) for v in _split_top(m.group(2)))
                w(("elif" if top[2][0] else "if") + f" {top[1]} in ({vals},):")
            top[2][0] = True
            ind += 1
            w("pass")
            continue
        if re.match(r"^end\s*select$", s):
            top = stack.pop()
            assert top[0] == "select", (sub.name, s)
            if top[2][0]:
                ind -= 1
            continue
        if s == "end":
            top = stack.pop()
            if top == "do" or top == "if" or (isinstance(top, tuple) and top[2][0]):
                ind -= 1
            continue
        stmt(s)
    assert not stack, (sub.name, stack)
    return "\n".join(out) + "\n"


def build(sources, globals_arrays, externals, trace=None, include_texts=None):
    """Translate every subroutine of the given source texts; returns {name: function}, the
    generated Python source and the include lines left out.  globals_arrays: module arrays
    (name -> numpy array, all lower bounds 1); externals: module scalars and the subroutines
    the sources call but do not define; include_texts: lower-cased include file name -> text
    spliced in where the sources include it."""
    py, names, includes = [], [], []
    SAVED_INIT.clear()
    ALLOC_DTYPE.clear()
    glb = {k: ["1"] * _np.ndim(v) for k, v in globals_arrays.items()}
    for text in sources:
        subs, inc = split_subroutines(logical_lines(text), include_texts)
        includes += inc
        for sub in subs:
            py.append(translate_subroutine(sub, glb, trace))
            names.append(sub.name)
    inits = []
    for gname, init in SAVED_INIT.items():
        inits.append("%s = %s" % (gname, "None" if init is None else emit(parse_expr(init), Scope({}))))
    src = "\n".join(inits) + "\n\n" + "\n".join(py)
    ns = {"_np": _np, "_div": _div, "_modulo": _modulo, "_mod": _mod, "_max": _max, "_min": _min,
          "_frange": _frange, "_sum": _sum, "_r4": _r4, "_trace": trace if trace is not None else []}
    ns.update({_pyname(k): v for k, v in globals_arrays.items()})
    ns.update({_pyname(k): v for k, v in externals.items()})
    exec(compile(src, "<fortran_subset>", "exec"), ns)
    return {n: ns[_pyname(n)] for n in names}, src, includes
