"""Fortran-subset translator -- TEST INFRASTRUCTURE ONLY.

This image has no Fortran compiler, so the reference's own Fortran routines
cannot be compiled.  This module translates the subset of Fortran 90 that
pyOM2's external-mode sources use (for_src/external/*.f90, the serial
parallel layer for_src/parallel/parallel_none.f90, for_src/main/
main_module.f90 and the grid/topography routines of for_src/main/
numerics.f90) into Python and runs it, so golden vectors can be produced from
the reference's source text itself.  tests/golden/make_ref_golden.py drives
it; the C oracle (pyom_oracle.c) is then checked against those vectors.

Semantics kept from Fortran (gfortran on x86-64, no FMA contraction):
  * types: integer (Python int), real*8 (numpy float64), default real
    (numpy float32: literals such as ``1.e-10`` or ``0.5`` are single
    precision and are promoted exactly where they meet a real*8), logical;
    mixed arithmetic promotes as Fortran does; integer division truncates
    toward zero; ``x**n`` with an integer n is a product of n factors;
    assignment converts to the target's type (real -> integer truncates);
  * arrays: column-major numpy arrays with their declared lower bounds;
    sections and whole-array expressions map onto numpy slicing; dummy
    arrays associate with the actual argument's storage (sequence
    association for explicit-shape dummies), so callees update the caller's
    arrays in place; scalar arguments are passed by reference (the callee's
    final value is written back to a variable or array element);
  * DO loops run their trip count and leave the index one step past the
    last value; EXIT/CYCLE (named or not), DO WHILE, block and logical IF,
    GOTO to statements at the top level of a routine, SAVE (explicit or by
    initialisation), module variables, COMMON blocks, PARAMETERs, implicit
    typing, ALLOCATE, WHERE, array constructors;
  * PRINT and WRITE statements are skipped (no output); a call of halt_stop
    raises ``HaltStop``.

Anything outside this subset raises ``F90Error`` at translation time rather
than being guessed.
"""
from __future__ import annotations

import math
import re

import numpy as np


class F90Error(Exception):
    pass


class HaltStop(Exception):
    pass


# ============================================================== source text
def _strip_comment(line):
    q = None
    for k, ch in enumerate(line):
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == "!":
            return line[:k]
    return line


def _split_top(s, sep):
    """Split at sep outside quotes and brackets."""
    out, depth, q, cur = [], 0, None, []
    k = 0
    while k < len(s):
        ch = s[k]
        if q:
            cur.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            cur.append(ch)
        elif ch in "([":
            depth += 1
            cur.append(ch)
        elif ch in ")]":
            depth -= 1
            cur.append(ch)
        elif depth == 0 and s.startswith(sep, k):
            out.append("".join(cur))
            cur = []
            k += len(sep)
            continue
        else:
            cur.append(ch)
        k += 1
    out.append("".join(cur))
    return out


def _lower_outside_quotes(s):
    out, q = [], None
    for ch in s:
        if q:
            out.append(ch)
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
            out.append(ch)
        else:
            out.append(ch.lower())
    return "".join(out)


def read_statements(text, fname="?"):
    """[(label, statement, line number)] of free-form source text."""
    stmts, buf, start = [], "", None
    for n, raw in enumerate(text.split("\n"), 1):
        line = _strip_comment(raw).rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if buf and s.startswith("&"):
            s = s[1:]
        if start is None:
            start = n
        if s.endswith("&"):
            buf += s[:-1] + " "
            continue
        full = buf + s
        buf = ""
        for part in _split_top(full, ";"):
            part = part.strip()
            if not part:
                continue
            m = re.match(r"^(\d+)\s+(.*)$", part)
            label = None
            if m:
                label, part = int(m.group(1)), m.group(2)
            stmts.append((label, _lower_outside_quotes(part).strip(), f"{fname}:{start}"))
        start = None
    return stmts


# ============================================================== expressions
_DOTOPS = {".and.", ".or.", ".not.", ".eqv.", ".neqv.", ".eq.", ".ne.", ".lt.", ".le.", ".gt.", ".ge.",
           ".true.", ".false."}
_TOK = re.compile(r"""
   (?P<ws>\s+)
 | (?P<str>'[^']*'|"[^"]*")
 | (?P<num>(\d+\.\d*|\.\d+|\d+)([edED][+-]?\d+)?(_\d+)?)
 | (?P<dot>\.[a-z]+\.)
 | (?P<name>[a-z_][a-z0-9_]*)
 | (?P<op>\*\*|//|==|/=|<=|>=|\(/|/\)|[-+*/()<>,:=%])
""", re.X)


def tokenize(s):
    toks, k = [], 0
    while k < len(s):
        m = _TOK.match(s, k)
        if not m:
            raise F90Error(f"cannot tokenize {s[k:]!r} in {s!r}")
        kind = m.lastgroup
        text = m.group(kind)
        if kind == "num":
            # 1.eq.2: the number ends before a dot operator
            mm = re.match(r"(\d+)\.([a-z]+)\.", s[k:])
            if mm and "." + mm.group(2) + "." in _DOTOPS:
                text = mm.group(1)
                toks.append(("num", text))
                k += len(text)
                continue
        if kind != "ws":
            if kind == "dot" and text not in _DOTOPS:
                raise F90Error(f"unknown operator {text}")
            toks.append((kind, text))
        k = m.end()
    return toks


class P:
    """Precedence-climbing parser over one expression's tokens."""

    BIN = [(".eqv.", ".neqv."), (".or.",), (".and.",), ("NOT",),
           ("==", "/=", "<", "<=", ">", ">=", ".eq.", ".ne.", ".lt.", ".le.", ".gt.", ".ge."), ("//",),
           ("+", "-"), ("*", "/"), ("**",)]
    REL = {".eq.": "==", ".ne.": "/=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}

    def __init__(self, s):
        self.t = tokenize(s)
        self.k = 0
        self.src = s

    def peek(self, off=0):
        return self.t[self.k + off] if self.k + off < len(self.t) else (None, None)

    def take(self, text=None):
        tok = self.peek()
        if text is not None and tok[1] != text:
            raise F90Error(f"expected {text!r} at {tok} in {self.src!r}")
        self.k += 1
        return tok

    def done(self):
        return self.k >= len(self.t)

    def expr(self, level=0):
        if level == len(self.BIN):
            return self.primary()
        ops = self.BIN[level]
        if ops == ("NOT",):
            if self.peek()[1] == ".not.":
                self.take()
                return ("un", ".not.", self.expr(level))
            return self.expr(level + 1)
        if ops == ("+", "-") and self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            left = ("un", op, self.expr(level + 1))
        elif ops == ("**",):
            left = self.primary()
            if self.peek()[1] == "**":
                self.take()
                right = self.expr(level - 1 if False else level)  # right associative, unary minus allowed
                return ("bin", "**", left, right)
            return left
        else:
            left = self.expr(level + 1)
        while self.peek()[1] in ops:
            op = self.take()[1]
            op = self.REL.get(op, op)
            if ops == ("+", "-") or ops == ("*", "/"):
                right = self.expr(level + 1)
            else:
                right = self.expr(level + 1)
            left = ("bin", op, left, right)
        return left

    def primary(self):
        kind, text = self.peek()
        if kind == "op" and text in ("+", "-"):  # unary sign after * or **
            self.take()
            return ("un", text, self.expr(len(self.BIN) - 2))
        if kind == "num":
            self.take()
            return ("num", text)
        if kind == "str":
            self.take()
            return ("str", text[1:-1])
        if kind == "dot" and text in (".true.", ".false."):
            self.take()
            return ("log", text == ".true.")
        if text == "(/":
            self.take()
            items = []
            while self.peek()[1] != "/)":
                items.append(self.expr())
                if self.peek()[1] == ",":
                    self.take()
            self.take("/)")
            return ("arr", items)
        if text == "(":
            self.take()
            e = self.expr()
            self.take(")")
            return ("paren", e)
        if kind == "name":
            self.take()
            if self.peek()[1] == "(":
                self.take()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.arg())
                        if self.peek()[1] == ",":
                            self.take()
                            continue
                        break
                self.take(")")
                return ("ref", text, args)
            return ("name", text)
        raise F90Error(f"unexpected {self.peek()} in {self.src!r}")

    def arg(self):
        # keyword argument, section triplet or expression
        if self.peek()[0] == "name" and self.peek(1)[1] == "=":
            name = self.take()[1]
            self.take("=")
            return ("kw", name, self.expr())
        lo = hi = st = None
        if self.peek()[1] != ":":
            lo = self.expr()
            if self.peek()[1] != ":":
                return lo
        self.take(":")
        if self.peek()[1] not in (",", ")", ":"):
            hi = self.expr()
        if self.peek()[1] == ":":
            self.take()
            st = self.expr()
        return ("sec", lo, hi, st)


def parse_arg(s):
    p = P(s)
    a = p.arg()
    if not p.done():
        raise F90Error(f"trailing tokens in argument {s!r}")
    return a


def parse_expr(s):
    p = P(s)
    e = p.expr()
    if not p.done():
        raise F90Error(f"trailing tokens in {s!r}: {p.t[p.k:]}")
    return e


# ============================================================== runtime
class FArray:
    """A Fortran array: column-major ndarray and per-dimension lower bounds."""
    __slots__ = ("a", "lo")

    def __init__(self, a, lo):
        self.a = a
        self.lo = tuple(int(v) for v in lo)


class GotoL(Exception):
    def __init__(self, label):
        self.label = label


class ExitL(Exception):
    def __init__(self, name, cycle=False):
        self.name = name
        self.cycle = cycle


DT = {"i": np.int64, "r4": np.float32, "r8": np.float64, "l": np.bool_, "c": object}


def cvt(t, v):
    """Assignment conversion to scalar type t."""
    if t == "r8":
        return np.float64(v)
    if t == "r4":
        return np.float32(v)
    if t == "i":
        if isinstance(v, (bool, np.bool_)):
            raise F90Error("logical assigned to integer")
        return int(v)  # truncation toward zero
    if t == "l":
        return bool(v)
    return v


def idiv(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
        a, b = int(a), int(b)
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q
    return a / b


def ipow(x, n):
    n = int(n)
    if n < 0:
        return 1 / ipow(x, -n)
    if n == 0:
        return type(x)(1) if not isinstance(x, np.ndarray) else np.ones_like(x)
    r = x
    for _ in range(n - 1):
        r = r * x
    return r


def alloc(t, bounds):
    lo = [int(b[0]) for b in bounds]
    shape = [max(0, int(b[1]) - int(b[0]) + 1) for b in bounds]
    return FArray(np.zeros(shape, dtype=DT[t], order="F"), lo)


def sec(X, subs):
    """Section or element view of FArray X; subs: int or (lo, hi, step)."""
    idx = []
    rank = 0
    for d, s in enumerate(subs):
        base = X.lo[d]
        ext = X.a.shape[d]
        if isinstance(s, tuple):
            lo, hi, st = s
            lo = base if lo is None else int(lo)
            hi = base + ext - 1 if hi is None else int(hi)
            st = 1 if st is None else int(st)
            a, b = lo - base, hi - base
            if st > 0:
                idx.append(slice(a, b + 1 if b + 1 > a else a, st))
            else:
                stop = b - 1
                idx.append(slice(a, None if stop < 0 else stop, st))
            rank += 1
        else:
            i = int(s) - base
            if i < 0 or i >= ext:
                raise F90Error(f"index {s} out of bounds {base}..{base + ext - 1}")
            idx.append(i)
    v = X.a[tuple(idx)]
    return FArray(v, [1] * rank) if rank else v


def elem_seq(X, subs):
    """Sequence association of an array element: the storage from X(subs) on."""
    off = 0
    mul = 1
    for d, s in enumerate(subs):
        off += (int(s) - X.lo[d]) * mul
        mul *= X.a.shape[d]
    flat = X.a.reshape(-1, order="F")
    if not np.shares_memory(flat, X.a):
        raise F90Error("element association on non-contiguous storage")
    return FArray(flat[off:], [1])


def dummy(actual, t, bounds, name):
    """Associate a dummy array with its actual argument.  bounds: list of
    (lo, hi) (hi None: assumed size / shape)."""
    if not isinstance(actual, FArray):
        if actual is None:
            raise F90Error(f"dummy {name}: no actual array")
        actual = FArray(np.atleast_1d(np.asarray(actual)), [1])
    a = actual.a
    if any(b[1] is None for b in bounds):  # assumed shape (:) or assumed size (*)
        if len(bounds) == a.ndim:
            return FArray(a, [1 if b[0] is None else b[0] for b in bounds])
        if len(bounds) == 1:  # assumed size
            flat = a.reshape(-1, order="F")
            return FArray(flat, [1 if bounds[0][0] is None else bounds[0][0]])
        raise F90Error(f"dummy {name}: rank mismatch")
    shape = tuple(max(0, int(h) - int(l) + 1) for l, h in bounds)
    lo = [int(l) for l, _ in bounds]
    if a.shape == shape:
        return FArray(a, lo)
    n = int(np.prod(shape))
    flat = a.reshape(-1, order="F")
    if not np.shares_memory(flat, a) and a.size > 1:
        raise F90Error(f"dummy {name}: sequence association with non-contiguous actual")
    if flat.size < n:
        raise F90Error(f"dummy {name}: actual has {flat.size} elements, dummy needs {n}")
    return FArray(flat[:n].reshape(shape, order="F"), lo)


def where_assign(target, mask, value):
    with np.errstate(all="ignore"):
        np.copyto(target, value, where=np.asarray(mask, dtype=bool), casting="unsafe")


def fmax(*a):
    r = a[0]
    for x in a[1:]:
        if isinstance(r, np.ndarray) or isinstance(x, np.ndarray):
            r = np.maximum(r, x)
        else:
            r = x if x > r else r
    return _promote(r, a)


def fmin(*a):
    r = a[0]
    for x in a[1:]:
        if isinstance(r, np.ndarray) or isinstance(x, np.ndarray):
            r = np.minimum(r, x)
        else:
            r = x if x < r else r
    return _promote(r, a)


def _promote(r, a):
    if isinstance(r, np.ndarray):
        return r
    if any(isinstance(x, np.float64) for x in a):
        return np.float64(r)
    if any(isinstance(x, np.float32) for x in a):
        return np.float32(r)
    return r


def fsign(a, b):
    if isinstance(a, (int, np.integer)) and not isinstance(a, np.floating):
        return abs(int(a)) if b >= 0 else -abs(int(a))
    return type(a)(abs(a)) if b >= 0 else type(a)(-abs(a))


def fmod(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
        return int(math.fmod(int(a), int(b)))
    return np.fmod(a, b)


def fnint(x):
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


# ============================================================== translator
_TYPES = r"(integer(?:\*\d+)?|real\s*\*\s*8|real\s*\(\s*kind\s*=\s*8\s*\)|real\s*\(\s*8\s*\)|double\s+precision|real(?:\*4)?|logical|character(?:\s*\*\s*\(?\s*[\w*]+\s*\)?|\s*\(\s*len\s*=\s*[\w*]+\s*\))?)"


def _norm_type(t):
    t = re.sub(r"\s+", "", t)
    if t.startswith("integer"):
        return "i"
    if t in ("real*8", "real(kind=8)", "real(8)", "doubleprecision"):
        return "r8"
    if t in ("real", "real*4"):
        return "r4"
    if t == "logical":
        return "l"
    if t.startswith("character"):
        return "c"
    raise F90Error(f"type {t}")


class Sym:
    def __init__(self, name, t=None, dims=None):
        self.name = name
        self.t = t
        self.dims = dims         # None (scalar) or list of (lo_expr, hi_expr) ASTs, or ':'/'*' markers
        self.alloc = False
        self.save = False
        self.param = None        # AST of a PARAMETER value
        self.init = None         # AST of an initial value (implies SAVE)
        self.dummy = False
        self.external = False
        self.common = None       # (block, position)
        self.intent = None

    @property
    def is_array(self):
        return self.dims is not None


INTRINSICS = {"abs", "max", "min", "sqrt", "exp", "log", "sin", "cos", "tan", "atan", "asin", "acos", "sign",
              "mod", "int", "nint", "real", "dble", "float", "maxval", "minval", "sum", "size", "allocated",
              "huge", "tiny", "epsilon", "floor", "ceiling", "sinh", "cosh", "tanh", "log10", "atan2", "trim",
              "len_trim", "present", "any", "all", "count", "transfer", "merge"}


class Unit:
    def __init__(self, kind, name, args, rtype=None, result=None):
        self.kind = kind          # module / subroutine / function
        self.name = name
        self.args = args
        self.rtype = rtype
        self.result = result or name
        self.syms = {}
        self.uses = []
        self.implicit = "default"  # default / none / {letter: type}
        self.body = []            # executable statements (label, text, where)
        self.spec_done = False


class Program:
    """All translated units; run-time state (module variables, common blocks,
    SAVE'd locals) lives on this object."""

    def __init__(self):
        self.units = {}
        self.modules = {}
        self.order = []
        self.externals = {}   # name -> python callable(prog, *args) returning write-back tuple
        self.code = {}
        self.fns = {}
        self.state = {}       # module name -> dict of variables
        self.common = {}
        self.saved = {}

    # ------------------------------------------------------------ parsing
    def add_source(self, text, fname="?"):
        stmts = read_statements(text, fname)
        cur = None
        for label, s, where in stmts:
            m_end = re.match(r"^end(\s*(subroutine|function|module|program)(\s+\w+)?)?$", s)
            if cur is not None and m_end:
                self.units[cur.name] = cur
                if cur.kind == "module":
                    self.modules[cur.name] = cur
                self.order.append(cur.name)
                cur = None
                continue
            if cur is None:
                m = re.match(r"^module\s+(\w+)$", s)
                if m:
                    cur = Unit("module", m.group(1), [])
                    continue
                m = re.match(r"^subroutine\s+(\w+)\s*(\((.*)\))?$", s)
                if m:
                    args = [a.strip() for a in (m.group(3) or "").split(",") if a.strip()]
                    cur = Unit("subroutine", m.group(1), args)
                    continue
                m = re.match(r"^(" + _TYPES + r"\s+)?function\s+(\w+)\s*\((.*?)\)\s*(result\s*\(\s*(\w+)\s*\))?$", s)
                if m:
                    rtype = _norm_type(m.group(2)) if m.group(2) else None
                    args = [a.strip() for a in m.group(4).split(",") if a.strip()]
                    cur = Unit("function", m.group(3), args, rtype, m.group(6))
                    continue
                raise F90Error(f"{where}: statement outside a unit: {s}")
            if s == "contains":
                raise F90Error(f"{where}: CONTAINS is not in the subset")
            if not self._spec(cur, s, where):
                cur.body.append((label, s, where))
        if cur is not None:
            raise F90Error(f"unterminated unit {cur.name}")

    def _decl_entities(self, cur, t, attrs, ents, where):
        dims_attr = None
        flags = set()
        intent = None
        for a in attrs:
            a = a.strip()
            if not a:
                continue
            m = re.match(r"^dimension\s*\((.*)\)$", a)
            if m:
                dims_attr = self._dims(m.group(1))
                continue
            m = re.match(r"^intent\s*\((\w+)\)$", a)
            if m:
                intent = m.group(1)
                continue
            if a in ("allocatable", "save", "parameter", "external", "target", "pointer", "optional", "public",
                     "private"):
                flags.add(a)
                continue
            raise F90Error(f"{where}: attribute {a}")
        for e in _split_top(ents, ","):
            e = e.strip()
            if not e:
                continue
            m = re.match(r"^(\w+)\s*(\((.*?)\))?\s*(=\s*(.*))?$", e)
            if not m:
                raise F90Error(f"{where}: entity {e}")
            name = m.group(1)
            sym = cur.syms.get(name) or Sym(name)
            cur.syms[name] = sym
            if t is not None:
                sym.t = t
            if m.group(3) is not None:
                sym.dims = self._dims(m.group(3))
            elif dims_attr is not None:
                sym.dims = dims_attr
            if "allocatable" in flags or "pointer" in flags:
                sym.alloc = True
            if "save" in flags:
                sym.save = True
            if "external" in flags:
                sym.external = True
            if intent:
                sym.intent = intent
            if m.group(5) is not None:
                val = parse_expr(m.group(5))
                if "parameter" in flags:
                    sym.param = val
                else:
                    sym.init = val
                    sym.save = True

    def _dims(self, s):
        out = []
        for d in _split_top(s, ","):
            d = d.strip()
            if d == ":":
                out.append((None, None))
            elif d == "*":
                out.append((None, None))
            elif ":" in _split_top(d, ":")[0] or len(_split_top(d, ":")) > 1:
                lo, hi = _split_top(d, ":")
                lo = parse_expr(lo) if lo.strip() else None
                hi = None if hi.strip() in ("", "*") else parse_expr(hi)
                out.append((lo, hi))
            else:
                out.append((("num", "1"), parse_expr(d)))
        return out

    def _spec(self, cur, s, where):
        """Handle a specification statement; False for an executable one."""
        m = re.match(r"^use\s+(\w+)(\s*,.*)?$", s)
        if m:
            if m.group(2):
                raise F90Error(f"{where}: USE with a list")
            cur.uses.append(m.group(1))
            return True
        if s == "implicit none":
            cur.implicit = "none"
            return True
        m = re.match(r"^implicit\s+(.*)$", s)
        if m:
            mm = re.match(r"^" + _TYPES + r"\s*\(\s*([a-z\-,\s]+)\)$", m.group(1))
            if not mm:
                raise F90Error(f"{where}: {s}")
            t = _norm_type(mm.group(1))
            mp = {} if not isinstance(cur.implicit, dict) else cur.implicit
            for rng in mm.group(2).split(","):
                rng = rng.strip()
                a, b = (rng.split("-") + [rng])[:2]
                for c in range(ord(a.strip()), ord(b.strip()) + 1):
                    mp[chr(c)] = t
            cur.implicit = mp
            return True
        m = re.match(r"^" + _TYPES + r"\s*(,\s*(.*?))?\s*::\s*(.*)$", s)
        if m:
            t = _norm_type(m.group(1))
            attrs = _split_top(m.group(3) or "", ",") if m.group(3) else []
            self._decl_entities(cur, t, attrs, m.group(4), where)
            return True
        m = re.match(r"^" + _TYPES + r"\s+([a-z].*)$", s)
        if m and not re.match(r"^\w+\s*=", m.group(2)) and "function" not in s.split("(")[0]:
            self._decl_entities(cur, _norm_type(m.group(1)), [], m.group(2), where)
            return True
        m = re.match(r"^dimension\s+(.*)$", s)
        if m:
            self._decl_entities(cur, None, [], m.group(1), where)
            return True
        m = re.match(r"^parameter\s*\((.*)\)$", s)
        if m:
            for e in _split_top(m.group(1), ","):
                name, val = e.split("=", 1)
                name = name.strip()
                sym = cur.syms.get(name) or Sym(name)
                cur.syms[name] = sym
                sym.param = parse_expr(val)
            return True
        m = re.match(r"^common\s*/\s*(\w+)\s*/\s*(.*)$", s)
        if m:
            for k, e in enumerate(_split_top(m.group(2), ",")):
                name = e.strip()
                sym = cur.syms.get(name) or Sym(name)
                cur.syms[name] = sym
                sym.common = (m.group(1), k)
            return True
        m = re.match(r"^external\s+(.*)$", s)
        if m:
            for e in m.group(1).split(","):
                name = e.strip()
                sym = cur.syms.get(name) or Sym(name)
                cur.syms[name] = sym
                sym.external = True
            return True
        if s == "save":
            for sym in cur.syms.values():
                sym.save = True
            return True
        m = re.match(r"^(private|public)\b", s)
        if m:
            return True
        return False

    # ------------------------------------------------------------ symbols
    def implicit_type(self, unit, name):
        if isinstance(unit.implicit, dict):
            return unit.implicit.get(name[0], "i" if "i" <= name[0] <= "n" else "r4")
        if unit.implicit == "none":
            return None
        return "i" if "i" <= name[0] <= "n" else "r4"

    def lookup(self, unit, name):
        """('local', Sym) / ('module', modname, Sym) / ('func', unitname) /
        ('intrinsic', name) / ('ext', name) / None."""
        if name in unit.syms:
            sym = unit.syms[name]
            if sym.external and name in self.units:
                return ("func", name)
            if sym.external:
                return ("ext", name)
            if not sym.is_array and sym.param is None and name in self.units and \
                    self.units[name].kind == "function" and name != unit.name:
                return ("func", name)  # a function declared by its type only
            if unit.kind == "module":
                return ("module", unit.name, sym)
            return ("local", sym)
        for mname in self._all_uses(unit):
            mod = self.modules[mname]
            if name in mod.syms:
                return ("module", mname, mod.syms[name])
        if name in self.units and self.units[name].kind == "function":
            return ("func", name)
        if name in INTRINSICS:
            return ("intrinsic", name)
        if name in self.externals:
            return ("ext", name)
        return None

    def _all_uses(self, unit):
        seen, out = set(), []

        def rec(u):
            for m in u.uses:
                if m not in seen:
                    if m not in self.modules:
                        raise F90Error(f"unknown module {m}")
                    seen.add(m)
                    out.append(m)
                    rec(self.modules[m])
        rec(unit)
        return out

    # ------------------------------------------------------------ compile
    def compile(self):
        self.failed = {}
        for name in self.order:
            u = self.units[name]
            if u.kind == "module":
                continue
            try:
                src = Gen(self, u).routine()
            except F90Error as e:
                # outside the subset (or calling routines that are not loaded): it fails
                # when it is called, not before
                self.failed[name] = str(e)
                self.fns[name] = (lambda msg: (lambda *a: (_ for _ in ()).throw(F90Error(msg))))(str(e))
                continue
            self.code[name] = src
            ns = {"RT": _RT, "np": np, "math": math, "PROG": self}
            try:
                exec(compile(src, f"<f90:{name}>", "exec"), ns)
            except SyntaxError as e:
                raise F90Error(f"generated code for {name} does not compile: {e}\n{src}")
            self.fns[name] = ns["R_" + name]
        for name in self.order:
            if self.units[name].kind == "module":
                self.init_module(name)

    def init_module(self, name):
        u = self.modules[name]
        st = self.state.setdefault(name, {})
        g = Gen(self, u)
        for sname, sym in u.syms.items():
            if sym.param is not None:
                st[sname] = g.const(sym)
        for sname, sym in u.syms.items():
            if sym.param is not None:
                continue
            if sym.is_array:
                if sym.alloc:
                    st[sname] = None
                else:
                    bounds = [(g.const_expr(lo) if lo is not None else 1, g.const_expr(hi)) for lo, hi in sym.dims]
                    st[sname] = alloc(sym.t, bounds)
            else:
                st[sname] = cvt(sym.t, g.const_expr(sym.init)) if sym.init is not None else cvt(sym.t, 0)

    def call(self, name, *args):
        """Run a translated routine (or function) with Python arguments;
        FArray / numpy arguments are updated in place.  Returns the function
        result, or the tuple of final scalar-argument values."""
        fn = self.fns[name]
        return fn(*args)

    def var(self, module, name):
        return self.state[module][name]

    def set(self, module, name, value):
        u = self.modules[module]
        sym = u.syms[name]
        if sym.is_array:
            if isinstance(value, FArray):
                self.state[module][name] = value
            else:
                cur = self.state[module][name]
                cur.a[...] = value
        else:
            self.state[module][name] = cvt(sym.t, value)


class _RTNS:
    pass


_RT = _RTNS()
for _n in ("FArray", "GotoL", "ExitL", "cvt", "idiv", "ipow", "alloc", "sec", "elem_seq", "dummy", "where_assign",
           "fmax", "fmin", "fsign", "fmod", "fnint", "HaltStop", "F90Error"):
    setattr(_RT, _n, globals()[_n])


class Gen:
    """Python code of one routine."""

    def __init__(self, prog, unit):
        self.p = prog
        self.u = unit
        self.lines = []
        self.ind = 1
        self.tmp = 0
        self.loops = []  # stack of (name or None)
        self.labels = set()

    # ------------------------------------------------------------ names
    def ref(self, name):
        """Python lvalue/rvalue of a variable and its Sym."""
        u = self.u
        if u.kind == "function" and name == u.result:
            sym = u.syms.get(name) or Sym(name, u.rtype or self.p.implicit_type(u, name))
            if sym.t is None:
                sym.t = u.rtype or self.p.implicit_type(u, name)
            u.syms[name] = sym
            return "v_" + name, sym
        r = self.p.lookup(u, name)
        if r is None:
            t = self.p.implicit_type(u, name)
            if t is None:
                raise F90Error(f"{u.name}: undeclared {name}")
            sym = Sym(name, t)
            u.syms[name] = sym
            r = ("local", sym)
        if r[0] == "local":
            sym = r[1]
            if sym.t is None:
                sym.t = self.p.implicit_type(u, name)
                if sym.t is None:
                    raise F90Error(f"{u.name}: untyped {name}")
            if sym.common is not None:
                return f"PROG.common[{sym.common[0]!r}][{sym.common[1]}]", sym
            if sym.save or (sym.alloc and not sym.dummy):
                return f"SV[{name!r}]", sym
            return "v_" + name, sym
        if r[0] == "module":
            return f"PROG.state[{r[1]!r}][{name!r}]", r[2]
        raise F90Error(f"{u.name}: {name} is not a variable ({r[0]})")

    # ------------------------------------------------------------ expressions
    def ex(self, e):
        """(code, type, rank) of an expression; arrays evaluate to ndarrays."""
        k = e[0]
        if k == "num":
            s = e[1]
            if re.fullmatch(r"\d+(_\d+)?", s):
                return s.split("_")[0], "i", 0
            kind8 = "d" in s or s.endswith("_8")
            body = s.split("_")[0].replace("d", "e")
            return (f"np.float64({body!r})" if kind8 else f"np.float32({body!r})"), ("r8" if kind8 else "r4"), 0
        if k == "str":
            return repr(e[1]), "c", 0
        if k == "log":
            return ("True" if e[1] else "False"), "l", 0
        if k == "paren":
            c, t, r = self.ex(e[1])
            return f"({c})", t, r
        if k == "arr":
            parts = [self.ex(x) for x in e[1]]
            t = self.promote([p[1] for p in parts])
            return f"np.array([{', '.join(p[0] for p in parts)}], dtype=RT_DT[{t!r}])", t, 1
        if k == "un":
            c, t, r = self.ex(e[2])
            if e[1] == ".not.":
                return (f"np.logical_not({c})" if r else f"(not {c})"), "l", r
            return f"({e[1]}{c})", t, r
        if k == "bin":
            return self.binop(e)
        if k == "name":
            name = e[1]
            code, sym = self.ref(name)
            if sym.param is not None and not sym.is_array:
                return code, sym.t, 0
            if sym.is_array:
                return f"{code}.a", sym.t, len(sym.dims)
            return code, sym.t, 0
        if k == "ref":
            return self.refexpr(e)
        raise F90Error(f"expression {e}")

    def promote(self, ts):
        if any(t == "r8" for t in ts):
            return "r8"
        if any(t == "r4" for t in ts):
            return "r4"
        if all(t == "l" for t in ts):
            return "l"
        return "i"

    def binop(self, e):
        _, op, a, b = e
        ca, ta, ra = self.ex(a)
        cb, tb, rb = self.ex(b)
        r = max(ra, rb)
        if op in (".and.", ".or."):
            if r:
                return f"np.logical_{op[1:-1]}({ca}, {cb})", "l", r
            return f"({ca} {op[1:-1]} {cb})", "l", 0
        if op in (".eqv.", ".neqv."):
            return f"(({ca}) {'==' if op == '.eqv.' else '!='} ({cb}))", "l", r
        if op in ("==", "/=", "<", "<=", ">", ">="):
            pop = {"/=": "!="}.get(op, op)
            return f"({ca} {pop} {cb})", "l", r
        if op == "//":
            return f"({ca} + {cb})", "c", 0
        t = self.promote([ta, tb])
        if op == "**":
            if tb == "i":
                return f"RT.ipow({ca}, {cb})", ta, r
            return f"({ca} ** {cb})", t, r
        if op == "/":
            if ta == "i" and tb == "i":
                if r:
                    raise F90Error("integer array division")
                return f"RT.idiv({ca}, {cb})", "i", 0
            return f"({ca} / {cb})", t, r
        return f"({ca} {op} {cb})", t, r

    def subs(self, args):
        """Python tuple of subscripts for RT.sec, and whether it is a section."""
        out, is_sec = [], False
        for a in args:
            if a[0] == "sec":
                is_sec = True
                lo = self.ex(a[1])[0] if a[1] is not None else "None"
                hi = self.ex(a[2])[0] if a[2] is not None else "None"
                st = self.ex(a[3])[0] if a[3] is not None else "None"
                out.append(f"({lo}, {hi}, {st})")
            else:
                c, t, r = self.ex(a)
                if r:
                    raise F90Error("vector subscript")
                out.append(c)
        return out, is_sec

    def elem(self, code, sym, args):
        idx = ", ".join(f"({self.ex(a)[0]}) - {code}.lo[{d}]" for d, a in enumerate(args))
        return f"{code}.a[{idx}]"

    def refexpr(self, e, as_actual=False):
        _, name, args = e
        u = self.u
        look = self.p.lookup(u, name) if not (u.kind == "function" and name == u.result and False) else None
        if look is None or look[0] in ("local", "module"):
            code, sym = self.ref(name)
            if not sym.is_array:
                raise F90Error(f"{u.name}: {name} is not an array")
            sub, is_sec = self.subs(args)
            if len(sub) != len(sym.dims):
                raise F90Error(f"{u.name}: rank of {name}")
            if is_sec:
                return f"RT.sec({code}, ({', '.join(sub)},)).a", sym.t, sum(1 for a in args if a[0] == "sec")
            if sym.t == "i":
                return f"int({self.elem(code, sym, args)})", "i", 0
            if sym.t == "l":
                return f"bool({self.elem(code, sym, args)})", "l", 0
            return self.elem(code, sym, args), sym.t, 0
        if look[0] == "intrinsic":
            return self.intrinsic(name, args)
        if look[0] == "func":
            fu = self.p.units[name]
            acts = [self.actual(a, fu, k)[0] for k, a in enumerate(args)]
            rt = fu.rtype or fu.syms.get(fu.result, Sym("", None)).t or self.p.implicit_type(fu, fu.result)
            return f"PROG.fns[{name!r}]({', '.join(acts)})", rt, 0
        if look[0] == "ext":
            acts = [self.actual(a, None, k)[0] for k, a in enumerate(args)]
            return f"PROG.externals[{name!r}](PROG, {', '.join(acts)})", "r8", 0
        raise F90Error(f"reference {name}")

    def intrinsic(self, name, args):
        xs = [self.ex(a) for a in args if a[0] != "kw"]
        kws = {a[1]: self.ex(a[2]) for a in args if a[0] == "kw"}
        c = [x[0] for x in xs]
        t0 = xs[0][1] if xs else None
        r = max([x[2] for x in xs] or [0])
        if name == "abs":
            return (f"np.abs({c[0]})" if r else f"abs({c[0]})"), t0, r
        if name in ("max", "min"):
            return f"RT.f{name}({', '.join(c)})", self.promote([x[1] for x in xs]), r
        if name in ("sqrt", "exp", "log", "sin", "cos", "tan", "atan", "asin", "acos", "sinh", "cosh", "tanh",
                    "log10"):
            fn = {"asin": "arcsin", "acos": "arccos", "atan": "arctan"}.get(name, name)
            if r:
                return f"np.{fn}({c[0]})", t0, r
            if t0 == "r4":
                return f"np.float32(np.{fn}({c[0]}))", "r4", 0
            return f"np.float64(math.{name}({c[0]}))", "r8", 0
        if name == "atan2":
            return f"np.float64(math.atan2({c[0]}, {c[1]}))", "r8", 0
        if name == "sign":
            return f"RT.fsign({c[0]}, {c[1]})", t0, 0
        if name == "mod":
            return f"RT.fmod({c[0]}, {c[1]})", self.promote([x[1] for x in xs]), 0
        if name == "int":
            return (f"({c[0]}).astype(np.int64)" if r else f"int({c[0]})"), "i", r
        if name == "nint":
            return f"RT.fnint({c[0]})", "i", 0
        if name in ("real", "float"):
            if "kind" in kws or len(c) > 1:
                return (f"np.float64({c[0]})" if not r else f"np.asarray({c[0]}, np.float64)"), "r8", r
            return (f"np.float32({c[0]})" if not r else f"np.asarray({c[0]}, np.float32)"), "r4", r
        if name == "dble":
            return (f"np.float64({c[0]})" if not r else f"np.asarray({c[0]}, np.float64)"), "r8", r
        if name in ("maxval", "minval"):
            return f"np.{'max' if name == 'maxval' else 'min'}({c[0]})", t0, 0
        if name == "sum":
            if "dim" in kws:
                raise F90Error("sum(dim=)")
            return f"RT.fsum({c[0]})", t0, 0
        if name == "size":
            if len(c) == 1 and "dim" not in kws:
                return f"np.size({c[0]})", "i", 0
            d = kws["dim"][0] if "dim" in kws else c[1]
            return f"np.shape({c[0]})[({d}) - 1]", "i", 0
        if name == "allocated":
            code, sym = self.ref(args[0][1])
            return f"({code} is not None)", "l", 0
        if name == "huge":
            return ("np.finfo(np.float64).max" if t0 == "r8" else "2147483647"), t0, 0
        if name == "any":
            return f"bool(np.any({c[0]}))", "l", 0
        if name == "all":
            return f"bool(np.all({c[0]}))", "l", 0
        if name == "count":
            return f"int(np.count_nonzero({c[0]}))", "i", 0
        if name == "merge":
            return f"({c[0]} if {c[2]} else {c[1]})", t0, 0
        raise F90Error(f"intrinsic {name}")

    def actual(self, a, fu, k):
        """Code of an actual argument passed to dummy k of unit fu (None:
        external); arrays pass as FArray, elements to array dummies by
        sequence association."""
        dsym = None
        if fu is not None and k < len(fu.args):
            dsym = fu.syms.get(fu.args[k])
        wants_array = dsym is not None and dsym.is_array
        if a[0] == "name":
            look = self.p.lookup(self.u, a[1])
            if look is not None and look[0] in ("local", "module"):
                code, sym = self.ref(a[1])
                if sym.is_array:
                    return code, True
            return self.ex(a)[0], False
        if a[0] == "ref":
            look = self.p.lookup(self.u, a[1])
            if look is not None and look[0] in ("local", "module"):
                code, sym = self.ref(a[1])
                if sym.is_array:
                    sub, is_sec = self.subs(a[2])
                    if is_sec:
                        return f"RT.sec({code}, ({', '.join(sub)},))", True
                    if wants_array or (fu is None and False):
                        return f"RT.elem_seq({code}, ({', '.join(sub)},))", True
        c, t, r = self.ex(a)
        if r:
            return f"RT.FArray({c}, [1] * np.ndim({c}))", True
        return c, False

    # ------------------------------------------------------------ statements
    def emit(self, s):
        self.lines.append("    " * self.ind + s)

    def const_expr(self, e):
        code = self.ex(e)[0]
        return eval(code, {"RT": _RT, "np": np, "math": math, "PROG": self.p, "RT_DT": DT, "SV": {}})

    def const(self, sym):
        v = self.const_expr(sym.param)
        return cvt(sym.t or self.p.implicit_type(self.u, sym.name), v)

    def assign(self, lhs, rhs_code, rhs_rank):
        """Statement assigning rhs to lhs (AST)."""
        if lhs[0] == "name":
            code, sym = self.ref(lhs[1])
            if sym.is_array:
                self.emit(f"{code}.a[...] = {rhs_code}")
            else:
                if rhs_rank:
                    raise F90Error("array assigned to scalar")
                self.emit(f"{code} = RT.cvt({sym.t!r}, {rhs_code})")
            return
        if lhs[0] == "ref":
            code, sym = self.ref(lhs[1])
            if not sym.is_array:
                raise F90Error(f"assignment to {lhs[1]}(...)")
            sub, is_sec = self.subs(lhs[2])
            if is_sec:
                self.emit(f"RT.sec({code}, ({', '.join(sub)},)).a[...] = {rhs_code}")
            else:
                self.emit(f"{self.elem(code, sym, lhs[2])} = {rhs_code}")
            return
        raise F90Error(f"assignment target {lhs}")

    def stmt(self, label, s, where, top=False):
        try:
            self._stmt(label, s, where, top)
        except F90Error as e:
            raise F90Error(f"{where}: {e} [{s}]") from None

    def _cond_split(self, s, kw):
        """(condition, rest) of 'kw (cond) rest'."""
        k = s.index("(")
        depth = 0
        for j in range(k, len(s)):
            if s[j] == "(":
                depth += 1
            elif s[j] == ")":
                depth -= 1
                if depth == 0:
                    return s[k + 1:j], s[j + 1:].strip()
        raise F90Error(f"unbalanced {s}")

    def _stmt(self, label, s, where, top):
        if re.match(r"^(print\b|write\s*\()", s):
            self.emit("pass")
            return
        if s == "continue":
            self.emit("pass")
            return
        if s == "return":
            self.emit(self.ret())
            return
        if re.match(r"^stop\b", s):
            self.emit("raise RT.HaltStop('stop')")
            return
        m = re.match(r"^go\s*to\s+(\d+)$", s)
        if m:
            self.emit(f"raise RT.GotoL({int(m.group(1))})")
            return
        m = re.match(r"^(exit|cycle)(\s+(\w+))?$", s)
        if m:
            name = m.group(3)
            if name is None or (self.loops and self.loops[-1] == name):
                if m.group(1) == "exit":
                    self.emit("break")
                else:
                    self.emit(self.cycle_code())
            else:
                self.emit(f"raise RT.ExitL({name!r}, {m.group(1) == 'cycle'})")
            return
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", s)
        if m:
            self.call(m.group(1), m.group(3) or "")
            return
        m = re.match(r"^(allocate|deallocate)\s*\((.*)\)$", s)
        if m:
            for ent in _split_top(m.group(2), ","):
                ent = ent.strip()
                mm = re.match(r"^(\w+)\s*(\((.*)\))?$", ent)
                code, sym = self.ref(mm.group(1))
                if m.group(1) == "deallocate":
                    self.emit(f"{code} = None")
                    continue
                bounds = []
                for d in _split_top(mm.group(3), ","):
                    parts = _split_top(d, ":")
                    if len(parts) == 2:
                        bounds.append(f"({self.ex(parse_expr(parts[0]))[0]}, {self.ex(parse_expr(parts[1]))[0]})")
                    else:
                        bounds.append(f"(1, {self.ex(parse_expr(parts[0]))[0]})")
                self.emit(f"{code} = RT.alloc({sym.t!r}, [{', '.join(bounds)}])")
            return
        if re.match(r"^where\s*\(", s):
            cond, rest = self._cond_split(s, "where")
            if not rest:
                raise F90Error("block WHERE")
            lhs, rhs = _split_top(rest, "=")
            tgt = parse_expr(lhs)
            cc = self.ex(parse_expr(cond))[0]
            rc = self.ex(parse_expr(rhs))[0]
            if tgt[0] == "name":
                code, sym = self.ref(tgt[1])
                tcode = f"{code}.a"
            else:
                code, sym = self.ref(tgt[1])
                sub, _ = self.subs(tgt[2])
                tcode = f"RT.sec({code}, ({', '.join(sub)},)).a"
            # the right-hand side is evaluated everywhere and kept where the mask holds
            self.emit("with np.errstate(all='ignore'):")
            self.emit(f"    RT.where_assign({tcode}, {cc}, {rc})")
            return
        if re.match(r"^if\s*\(", s):
            cond, rest = self._cond_split(s, "if")
            cc = self.ex(parse_expr(cond))[0]
            if rest == "then":
                raise F90Error("block IF handled by the block parser")
            self.emit(f"if {cc}:")
            self.ind += 1
            self.stmt(None, rest, where)
            self.ind -= 1
            return
        # assignment
        parts = _split_top(s, "=")
        parts = [p for p in parts]
        if len(parts) >= 2:
            # rejoin comparison operators split by '='
            lhs = parts[0]
            rhs = "=".join(parts[1:])
            if lhs.strip() and not lhs.rstrip().endswith(("<", ">", "/", "=")) and not rhs.startswith("="):
                L = parse_expr(lhs.strip())
                R = parse_expr(rhs.strip())
                rc, rt, rr = self.ex(R)
                self.assign(L, rc, rr)
                return
        raise F90Error(f"statement not in the subset: {s}")

    def call(self, name, argtext):
        args = [parse_arg(a) for a in _split_top(argtext, ",")] if argtext.strip() else []
        if name == "halt_stop" and name not in self.p.units:
            self.emit("raise RT.HaltStop('halt_stop')")
            return
        fu = self.p.units.get(name)
        if fu is None:
            if name not in self.p.externals:
                raise F90Error(f"call of unknown routine {name}")
            acts = [self.actual(a, None, k) for k, a in enumerate(args)]
            t = self.tmpname()
            self.emit(f"{t} = PROG.externals[{name!r}](PROG, {', '.join(c for c, _ in acts)})")
            self.writeback(t, args, acts)
            return
        if len(args) != len(fu.args):
            raise F90Error(f"call {name}: {len(args)} arguments for {len(fu.args)}")
        acts = [self.actual(a, fu, k) for k, a in enumerate(args)]
        t = self.tmpname()
        self.emit(f"{t} = PROG.fns[{name!r}]({', '.join(c for c, _ in acts)})")
        self.writeback(t, args, acts)

    def writeback(self, t, args, acts):
        for k, (a, (c, is_arr)) in enumerate(zip(args, acts)):
            if is_arr:
                continue
            if a[0] == "name":
                look = self.p.lookup(self.u, a[1])
                if look is None or look[0] in ("local", "module"):
                    code, sym = self.ref(a[1])
                    if sym.param is None and not sym.is_array:
                        self.emit(f"if {t} is not None and {t}[{k}] is not None: {code} = RT.cvt({sym.t!r}, {t}[{k}])")
            elif a[0] == "ref":
                look = self.p.lookup(self.u, a[1])
                if look is not None and look[0] in ("local", "module"):
                    code, sym = self.ref(a[1])
                    if sym.is_array:
                        sub, is_sec = self.subs(a[2])
                        if not is_sec:
                            self.emit(f"if {t} is not None and {t}[{k}] is not None: "
                                      f"{self.elem(code, sym, a[2])} = {t}[{k}]")

    def tmpname(self):
        self.tmp += 1
        return f"_t{self.tmp}"

    def ret(self):
        u = self.u
        if u.kind == "function":
            code, sym = self.ref(u.result)
            return f"return {code}"
        outs = []
        for a in u.args:
            sym = u.syms.get(a)
            if sym is not None and sym.is_array:
                outs.append("None")
            else:
                outs.append("v_" + a)
        return f"return ({', '.join(outs)}{',' if len(outs) == 1 else ''})"

    def cycle_code(self):
        return "continue"

    # ------------------------------------------------------------ blocks
    def block(self, stmts, top=False):
        """Emit a statement list with nested constructs."""
        k = 0
        while k < len(stmts):
            label, s, where = stmts[k]
            m_do = re.match(r"^((\w+)\s*:\s*)?do(\s+(.*))?$", s)
            if m_do:
                if re.match(r"^do\s+\d+", s):
                    raise F90Error(f"{where}: label-terminated DO")
                name = m_do.group(2)
                spec = (m_do.group(4) or "").strip()
                end = self.match_end(stmts, k, r"^((\w+)\s*:\s*)?do(\s+.*)?$", r"^end\s*do(\s+\w+)?$")
                self.do_loop(name, spec, stmts[k + 1:end], where)
                k = end + 1
                continue
            if re.match(r"^if\s*\(", s):
                cond, rest = self._cond_split(s, "if")
                if rest == "then":
                    end, branches = self.if_branches(stmts, k)
                    first = True
                    for c, body in branches:
                        if c is None:
                            self.emit("else:")
                        else:
                            cc = self.ex(parse_expr(c))[0]
                            self.emit(f"{'if' if first else 'elif'} {cc}:")
                        first = False
                        self.ind += 1
                        self.emit("pass")
                        self.block(body)
                        self.ind -= 1
                    k = end + 1
                    continue
            if re.match(r"^end\s*(do|if)\b", s) or re.match(r"^else\b", s):
                raise F90Error(f"{where}: unmatched {s}")
            self.stmt(label, s, where, top)
            k += 1

    def match_end(self, stmts, k, open_re, close_re):
        depth = 0
        for j in range(k, len(stmts)):
            s = stmts[j][1]
            if re.match(open_re, s):
                depth += 1
            elif re.match(close_re, s):
                depth -= 1
                if depth == 0:
                    return j
        raise F90Error(f"{stmts[k][2]}: no end for {stmts[k][1]}")

    def if_branches(self, stmts, k):
        depth = 0
        branches = []
        cur_cond = self._cond_split(stmts[k][1], "if")[0]
        cur = []
        for j in range(k + 1, len(stmts)):
            s = stmts[j][1]
            if re.match(r"^if\s*\(", s) and self._cond_split(s, "if")[1] == "then":
                depth += 1
                cur.append(stmts[j])
                continue
            if re.match(r"^end\s*if$", s):
                if depth == 0:
                    branches.append((cur_cond, cur))
                    return j, branches
                depth -= 1
                cur.append(stmts[j])
                continue
            if depth == 0 and re.match(r"^else\s*if\s*\(", s):
                branches.append((cur_cond, cur))
                cur_cond = self._cond_split(s, "else if" if "else if" in s else "elseif")[0]
                cur = []
                continue
            if depth == 0 and s == "else":
                branches.append((cur_cond, cur))
                cur_cond = None
                cur = []
                continue
            cur.append(stmts[j])
        raise F90Error(f"{stmts[k][2]}: no END IF")

    def do_loop(self, name, spec, body, where):
        self.loops.append(name)
        wrap = name is not None
        if wrap:
            self.emit("try:")
            self.ind += 1
        if spec == "":
            self.emit("while True:")
            self.ind += 1
            self.emit("pass")
            self.block(body)
            self.ind -= 1
        elif spec.startswith("while"):
            cond, rest = self._cond_split(spec, "while")
            self.emit(f"while {self.ex(parse_expr(cond))[0]}:")
            self.ind += 1
            self.emit("pass")
            self.block(body)
            self.ind -= 1
        else:
            m = re.match(r"^(\w+)\s*=\s*(.*)$", spec)
            var = m.group(1)
            bounds = _split_top(m.group(2), ",")
            lo = self.ex(parse_expr(bounds[0]))[0]
            hi = self.ex(parse_expr(bounds[1]))[0]
            st = self.ex(parse_expr(bounds[2]))[0] if len(bounds) > 2 else "1"
            code, sym = self.ref(var)
            n = self.tmpname()
            stv = self.tmpname()
            self.emit(f"{stv} = int({st})")
            self.emit(f"{code} = int({lo})")
            self.emit(f"{n} = max(0, RT.idiv(int({hi}) - {code} + {stv}, {stv}))")
            self.emit(f"while {n} > 0:")
            self.ind += 1
            # cycle: the increment runs first (the body is wrapped in a one-pass loop)
            self.emit(f"{n} -= 1")
            self.emit("for _once in (0,):")
            self.ind += 1
            self.emit("pass")
            inner = self.loops
            self.loops = inner[:-1] + [("__inner__", name)]
            self.block_do_body(body)
            self.loops = inner
            self.ind -= 1
            self.emit("else:")
            self.ind += 1
            self.emit(f"{code} = {code} + {stv}")
            self.emit("continue")
            self.ind -= 1
            # reached only by an EXIT (break out of the one-pass loop)
            self.emit("break")
            self.ind -= 1
        if wrap:
            self.ind -= 1
            self.emit("except RT.ExitL as _e:")
            self.ind += 1
            self.emit(f"if _e.name != {name!r} or _e.cycle: raise")
            self.ind -= 1
        self.loops.pop()

    def block_do_body(self, body):
        # inside the one-pass loop: EXIT -> break (leaves the one-pass loop without
        # the increment, then the outer while breaks); CYCLE -> continue of the
        # one-pass loop, which ends it normally (increment, next trip)
        self.block(body)

    # ------------------------------------------------------------ routine
    def routine(self):
        u = self.u
        body = u.body
        # labels that GOTOs target, at the top level
        targets = set()
        for _, s, _ in body:
            for m in re.finditer(r"go\s*to\s+(\d+)", s):
                targets.add(int(m.group(1)))
        top_labels = self.top_labels(body)
        for t in targets:
            if t not in top_labels:
                raise F90Error(f"{u.name}: GOTO {t} target not at the top level")
        head = [f"def R_{u.name}({', '.join('a_' + a for a in u.args)}):",
                "    RT_DT = DT_",
                f"    SV = PROG.saved.setdefault({u.name!r}, {{}})"]
        for a in u.args:
            sym = u.syms.get(a)
            if sym is None:
                sym = Sym(a, self.p.implicit_type(u, a))
                u.syms[a] = sym
            sym.dummy = True
        # the body first: implicitly typed locals become known while it is generated
        self.lines = []
        self.ind = 1
        self.body_code(body, targets)
        body_lines = self.lines
        self.lines = []
        self.ind = 1
        # dummies
        for a in u.args:
            sym = u.syms.get(a)
            if sym is None:
                t = self.p.implicit_type(u, a)
                sym = Sym(a, t)
                u.syms[a] = sym
            sym.dummy = True
            if sym.t is None:
                sym.t = self.p.implicit_type(u, a)
        # parameters and saved initial values
        for name, sym in u.syms.items():
            if sym.param is not None:
                if sym.t is None:
                    sym.t = self.p.implicit_type(u, name)
        for name, sym in u.syms.items():
            if sym.param is not None and not sym.is_array:
                self.emit(f"v_{name} = RT.cvt({sym.t!r}, {self.ex(sym.param)[0]})")
        for a in u.args:
            if not u.syms[a].is_array:
                self.emit(f"v_{a} = a_{a}")
        for a in u.args:
            sym = u.syms[a]
            if sym.is_array:
                bounds = []
                for lo, hi in sym.dims:
                    lo_c = self.ex(lo)[0] if lo is not None else "None"
                    hi_c = self.ex(hi)[0] if hi is not None else "None"
                    bounds.append(f"({lo_c}, {hi_c})")
                self.emit(f"v_{a} = RT.dummy(a_{a}, {sym.t!r}, [{', '.join(bounds)}], {a!r})")
        for name, sym in u.syms.items():
            if sym.dummy or sym.param is not None or sym.common is not None or sym.external:
                continue
            if u.kind == "function" and name == u.result:
                continue
            if self.p.lookup(u, name)[0] != "local":
                continue  # a function or external declared by its type
            if sym.t is None:
                sym.t = self.p.implicit_type(u, name)
                if sym.t is None:
                    continue
            code, _ = self.ref(name)
            if sym.save or (sym.alloc and sym.is_array):
                if sym.is_array and not sym.alloc:
                    bounds = ", ".join(f"({self.ex(lo)[0] if lo is not None else 1}, {self.ex(hi)[0]})"
                                       for lo, hi in sym.dims)
                    self.emit(f"if {name!r} not in SV: SV[{name!r}] = RT.alloc({sym.t!r}, [{bounds}])")
                elif sym.is_array:
                    self.emit(f"if {name!r} not in SV: SV[{name!r}] = None")
                else:
                    init = self.ex(sym.init)[0] if sym.init is not None else "0"
                    self.emit(f"if {name!r} not in SV: SV[{name!r}] = RT.cvt({sym.t!r}, {init})")
            elif sym.is_array:
                bounds = ", ".join(f"({self.ex(lo)[0] if lo is not None else 1}, {self.ex(hi)[0]})"
                                   for lo, hi in sym.dims)
                self.emit(f"{code} = RT.alloc({sym.t!r}, [{bounds}])")
            else:
                self.emit(f"{code} = RT.cvt({sym.t!r}, 0)")
        for name, sym in u.syms.items():
            if sym.common is not None:
                blk, pos = sym.common
                self.emit(f"PROG.common.setdefault({blk!r}, {{}}).setdefault({pos}, RT.cvt({sym.t or self.p.implicit_type(u, name)!r}, 0))")
        if u.kind == "function":
            code, sym = self.ref(u.result)
            self.emit(f"{code} = RT.cvt({sym.t!r}, 0)")
        src = "\n".join(head + self.lines + body_lines) + "\n"
        return src.replace("RT_DT = DT_", "RT_DT = RT.DT")

    def body_code(self, body, targets):
        u = self.u
        # body with GOTO segments
        if targets:
            segs = self.segments(body, targets)
            self.emit("_pc = 0")
            self.emit("while True:")
            self.ind += 1
            self.emit("try:")
            self.ind += 1
            for idx, (lab, seg) in enumerate(segs):
                self.emit(f"if _pc <= {idx}:")
                self.ind += 1
                self.emit("pass")
                self.block(seg, top=True)
                self.ind -= 1
            self.emit("break")
            self.ind -= 1
            self.emit("except RT.GotoL as _g:")
            self.ind += 1
            lm = {lab: idx for idx, (lab, _) in enumerate(segs) if lab is not None}
            self.emit(f"_pc = {lm!r}[_g.label]")
            self.ind -= 2
        else:
            self.block(body, top=True)
        self.emit(self.ret())

    def top_labels(self, body):
        labels = set()
        depth = 0
        for lab, s, _ in body:
            if lab is not None and depth == 0:
                labels.add(lab)
            if re.match(r"^((\w+)\s*:\s*)?do(\s+.*)?$", s) or \
                    (re.match(r"^if\s*\(", s) and self._cond_split(s, "if")[1] == "then"):
                depth += 1
            elif re.match(r"^end\s*(do|if)\b", s):
                depth -= 1
        return labels

    def segments(self, body, targets):
        segs, cur, lab = [], [], None
        for st in body:
            if st[0] in targets:
                segs.append((lab, cur))
                cur, lab = [], st[0]
            cur.append(st)
        segs.append((lab, cur))
        return segs


_RT.DT = DT


def fsum(a):
    """sum() of an array in Fortran's column-major order, accumulated
    sequentially as gfortran does without -ffast-math."""
    flat = np.asarray(a).reshape(-1, order="F")
    if flat.dtype.kind in "iub":
        return int(flat.sum())
    s = flat.dtype.type(0)
    for v in flat:
        s = s + v
    return s


_RT.fsum = fsum


def translate(paths, externals=None):
    """A compiled Program of the given Fortran source files."""
    prog = Program()
    for p in paths:
        with open(p) as fh:
            prog.add_source(fh.read(), p.split("/")[-1])
    if externals:
        prog.externals.update(externals)
    prog.compile()
    return prog
