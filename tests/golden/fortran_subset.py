"""Executes the reference's own Fortran source of the hot-path routines (test infrastructure).

The reference (GETM 2.5, Fortran 90 + cpp) cannot be compiled in this environment: no Fortran
compiler is installed. To pin the C++ oracle to the reference itself rather than to a reading of
it, this module runs the reference's .F90 files directly:

  1. the C preprocessor expands them exactly as GETM's build does (cppdefs.h: HALO=2, REALTYPE
     = real(kind=selected_real_kind(13)), Cartesian metrics DXU -> dx, ...; none of SPHERICAL,
     CURVILINEAR, GETM_PARALLEL, SLICE_MODEL, DEBUG, _POINTER_REMAP_ defined);
  2. a translator turns the Fortran 90 subset used by those routines (modules with parameters,
     derived types with pointer components, explicit-shape / pointer / allocatable arrays with
     arbitrary lower bounds, array sections and whole-array assignment, DO / DO WHILE / IF /
     SELECT CASE / CYCLE, optional arguments, intrinsic functions) into Python;
  3. the Python runs with IEEE double arithmetic (numpy float64 scalars, no fused multiply-add),
     evaluating every expression in Fortran's order with explicit parentheses; real literals
     without a d exponent are rounded to single precision first, as Fortran does.

Only tests/golden/make_golden.py imports this module, here where the reference is mounted; it
writes input/output fixtures that the test suite compares with the oracle. Nothing here runs on
the GPU machine. OpenMP directives are comments to the translator, so loops run sequentially
(every routine covered is written to give identical results under any OpenMP schedule).
"""
from __future__ import annotations

import math
import os
import re
import subprocess
import types

import numpy as np

REF = os.environ.get("GETM_REFERENCE", "/root/reference")


class FortranStop(RuntimeError):
    pass


# ------------------------------------------------------------------------------------------------
# runtime: arrays with Fortran bounds
class FArr:
    """Fortran array: numpy storage in column-major order plus lower bounds."""

    __slots__ = ("a", "lb")

    def __init__(self, a: np.ndarray, lb):
        self.a = a
        self.lb = tuple(int(x) for x in lb)

    @property
    def ub(self):
        return tuple(l + n - 1 for l, n in zip(self.lb, self.a.shape))

    def _idx(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        if len(key) != self.a.ndim:
            raise IndexError(f"rank mismatch {len(key)} vs {self.a.ndim}")
        out = []
        scalar = True
        for d, k in enumerate(key):
            l = self.lb[d]
            if isinstance(k, FSlice):
                lo = l if k.lo is None else int(k.lo)
                hi = self.lb[d] + self.a.shape[d] - 1 if k.hi is None else int(k.hi)
                if lo - l < 0 or hi - l >= self.a.shape[d]:
                    if hi >= lo:
                        raise IndexError(f"section {lo}:{hi} out of bounds dim {d} ({l}:{l + self.a.shape[d] - 1})")
                out.append(slice(lo - l, hi - l + 1))
                scalar = False
            else:
                i = int(k) - l
                if i < 0 or i >= self.a.shape[d]:
                    raise IndexError(f"index {int(k)} out of bounds dim {d} ({l}:{l + self.a.shape[d] - 1})")
                out.append(i)
        return tuple(out), scalar

    def __getitem__(self, key):
        idx, scalar = self._idx(key)
        v = self.a[idx]
        if scalar:
            return _scal(v)
        return v

    def section(self, key):
        """Array section as a new FArr (lower bounds 1) sharing storage."""
        idx, scalar = self._idx(key)
        v = self.a[idx]
        if scalar:
            return _scal(v)
        return FArr(v, (1,) * v.ndim)

    def __setitem__(self, key, val):
        idx, scalar = self._idx(key)
        if isinstance(val, FArr):
            val = val.a
        self.a[idx] = val

    def __array__(self, dtype=None, copy=None):
        return self.a if dtype is None else self.a.astype(dtype)


class FSlice:
    __slots__ = ("lo", "hi")

    def __init__(self, lo=None, hi=None):
        self.lo, self.hi = lo, hi


def _scal(v):
    if isinstance(v, np.bool_):
        return bool(v)
    if isinstance(v, (np.integer,)):
        return int(v)
    return v


KIND_DTYPE = {"real": np.float64, "integer": np.int64, "logical": np.bool_}


def _alloc(bounds, kind):
    lb = [int(b[0]) for b in bounds]
    shape = [max(0, int(b[1]) - int(b[0]) + 1) for b in bounds]
    return FArr(np.zeros(shape, dtype=KIND_DTYPE[kind], order="F"), lb)


def _bind(actual, bounds, kind):
    """Explicit-shape dummy argument: the actual's storage seen with the dummy's bounds
    (sequence association; the actual must be contiguous in column-major order)."""
    if actual is None:
        return None
    a = actual.a if isinstance(actual, FArr) else np.asarray(actual)
    lb = [int(b[0]) for b in bounds]
    shape = [int(b[1]) - int(b[0]) + 1 for b in bounds]
    n = int(np.prod(shape))
    if not (a.flags.f_contiguous or a.ndim <= 1):
        raise ValueError("non-contiguous actual argument")
    flat = a.reshape(-1, order="F")
    if flat.size < n:
        raise ValueError(f"actual too small for dummy ({flat.size} < {n})")
    if not np.shares_memory(flat, a) and a.size:
        raise ValueError("binding would copy")
    return FArr(flat[:n].reshape(shape, order="F"), lb)


def _assign(lhs, rhs):
    if isinstance(rhs, FArr):
        rhs = rhs.a
    lhs.a[...] = rhs


def _range(a, b, c=1):
    a, b, c = int(a), int(b), int(c)
    if c > 0:
        return range(a, b + 1, c)
    return range(a, b - 1, c)


def _div(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)) and not isinstance(a, bool):
        q = abs(int(a)) // abs(int(b))
        return q if (a >= 0) == (b >= 0) else -q
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        return np.float64(a) / np.float64(b) if not isinstance(a, np.ndarray) and not isinstance(b, np.ndarray) \
            else np.asarray(a, np.float64) / np.asarray(b, np.float64)


def _num(x):
    """Promote Python ints used in real arithmetic: keep as is (int op float64 -> float64)."""
    return x


def _powi(a, n):
    """x**n for a real x and a constant integer n as gfortran compiles it: multiplications
    (GCC expands __builtin_powi with a constant exponent into a chain of products: x*x for 2,
    (x*x)*x for 3, (x*x)*(x*x) for 4, square-and-multiply beyond), never a call of pow()."""
    if n < 0:
        return np.float64(1.0) / _powi(a, -n)
    if n == 0:
        return np.float64(1.0)
    if n == 1:
        return a
    if n == 2:
        return a * a
    if n == 3:
        return (a * a) * a
    half = _powi(a, n // 2)
    return half * half if n % 2 == 0 else (half * half) * a


def _pow(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)) and b >= 0:
        return int(a) ** int(b)
    with np.errstate(all="ignore"):
        if isinstance(b, (int, np.integer)) and not isinstance(b, bool):
            if isinstance(a, np.ndarray):
                return np.frompyfunc(lambda v: _powi(np.float64(v), int(b)), 1, 1)(a).astype(np.float64)
            return _powi(np.float64(a), int(b))
        if np.ndim(a) == 0 and np.ndim(b) == 0:
            try:
                return np.float64(math.pow(float(a), float(b)))  # the C library's pow, as gfortran calls it
            except (ValueError, OverflowError):
                pass
        return np.float64(a) ** b


def _arr(x):
    return x.a if isinstance(x, FArr) else x


def _cmp(op):
    def f(a, b):
        a, b = _arr(a), _arr(b)
        r = op(a, b)
        return bool(r) if np.ndim(r) == 0 else r
    return f


_eq = _cmp(lambda a, b: a == b)
_ne = _cmp(lambda a, b: a != b)
_lt = _cmp(lambda a, b: a < b)
_le = _cmp(lambda a, b: a <= b)
_gt = _cmp(lambda a, b: a > b)
_ge = _cmp(lambda a, b: a >= b)


def _and(a, b):
    a, b = _arr(a), _arr(b)
    if np.ndim(a) == 0 and np.ndim(b) == 0:
        return bool(a) and bool(b)
    return np.logical_and(a, b)


def _or(a, b):
    a, b = _arr(a), _arr(b)
    if np.ndim(a) == 0 and np.ndim(b) == 0:
        return bool(a) or bool(b)
    return np.logical_or(a, b)


def _not(a):
    a = _arr(a)
    return (not bool(a)) if np.ndim(a) == 0 else np.logical_not(a)


def _neg(a):
    a = _arr(a)
    return -a


def _bin(op):
    def f(a, b):
        a, b = _arr(a), _arr(b)
        with np.errstate(all="ignore"):
            return op(a, b)
    return f


_add = _bin(lambda a, b: a + b)
_sub = _bin(lambda a, b: a - b)
_mul = _bin(lambda a, b: a * b)


def _fmin(*xs):
    xs = [_arr(x) for x in xs]
    if all(np.ndim(x) == 0 for x in xs):
        r = xs[0]
        for x in xs[1:]:
            if x < r:
                r = x
        return r
    r = xs[0]
    for x in xs[1:]:
        r = np.where(x < r, x, r)
    return r


def _fmax(*xs):
    xs = [_arr(x) for x in xs]
    if all(np.ndim(x) == 0 for x in xs):
        r = xs[0]
        for x in xs[1:]:
            if x > r:
                r = x
        return r
    r = xs[0]
    for x in xs[1:]:
        r = np.where(x > r, x, r)
    return r


def _ceiling(x):
    x = _arr(x)
    r = np.ceil(x)
    return int(r) if np.ndim(r) == 0 else r.astype(np.int64)


def _floor(x):
    x = _arr(x)
    r = np.floor(x)
    return int(r) if np.ndim(r) == 0 else r.astype(np.int64)


def _abs(x):
    x = _arr(x)
    return abs(x) if np.ndim(x) == 0 else np.abs(x)


def _maxval(x):
    return _scal(np.max(_arr(x)))


def _minval(x):
    return _scal(np.min(_arr(x)))


def _sum(x):
    return _scal(np.sum(_arr(x)))


def _real(x, kind=None):
    x = _arr(x)
    return np.float64(x) if np.ndim(x) == 0 else np.asarray(x, np.float64)


def _int(x):
    x = _arr(x)
    return int(x) if np.ndim(x) == 0 else np.asarray(x).astype(np.int64)


def _mod(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
        return int(np.fmod(int(a), int(b)))
    return np.fmod(np.float64(a), np.float64(b))


def _sign(a, b):
    return abs(a) if b >= 0 else -abs(a)


def _libm(fn, x):
    """An elemental math function evaluated by the C library (math.exp / math.log call the
    platform libm, as gfortran's compiled code does; numpy's own vectorised exp and log can differ
    from it in the last bit)."""
    x = _arr(x)
    if np.ndim(x) == 0:
        try:
            return np.float64(fn(float(x)))
        except (ValueError, OverflowError):
            with np.errstate(all="ignore"):
                return np.float64(np.exp(x) if fn is math.exp else np.log(x))
    return np.frompyfunc(lambda v: _libm(fn, v), 1, 1)(x).astype(np.float64)


def _exp(x):
    return _libm(math.exp, x)


def _log(x):
    return _libm(math.log, x)


def _sqrt(x):
    return np.sqrt(_arr(x))


def _present(x):
    return x is not None


def _wassign(lhs, rhs, mask):
    """An assignment inside a WHERE construct: the elements of lhs where mask holds."""
    r = _arr(rhs)
    if np.ndim(r) == 0:
        lhs.a[mask] = r
    else:
        lhs.a[mask] = np.asarray(r)[mask]


class _Out(dict):
    """Final values of a subroutine's scalar dummy arguments, by position: the caller copies them
    back into actual arguments that are variables or array elements (Fortran passes by reference;
    the translated Python passes scalars by value)."""


class Counter:
    def __init__(self):
        self.writes = 0


WRITES = Counter()


def _write(*a):
    WRITES.writes += 1


INTRINSICS = {
    "abs": "_abs", "min": "_fmin", "max": "_fmax", "ceiling": "_ceiling", "floor": "_floor", "maxval": "_maxval",
    "minval": "_minval", "sum": "_sum", "real": "_real", "dble": "_real", "int": "_int", "mod": "_mod",
    "sign": "_sign", "exp": "_exp", "sqrt": "_sqrt", "present": "_present", "tanh": "np.tanh", "sin": "np.sin",
    "cos": "np.cos", "log": "_log", "selected_real_kind": "_srk", "allocated": "_allocated", "float": "_real",
    "huge": "_huge",
}


def _allocated(x):
    return x is not None


def _huge(x):
    return np.finfo(np.float64).max


def _srk(*a):
    return 8


# ------------------------------------------------------------------------------------------------
# front end
def preprocess(path: str, defines=()) -> str:
    cmd = ["cpp", "-traditional-cpp", "-P", f"-I{os.path.join(REF, 'include')}"] + [f"-D{d}" for d in defines] + [path]
    return subprocess.run(cmd, check=True, capture_output=True, text=True).stdout


def _strip_comment(line: str) -> str:
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


def statements(text: str):
    buf = ""
    for raw in text.splitlines():
        line = _strip_comment(raw).rstrip()
        if not line.strip():
            continue
        s = line.strip()
        if buf:
            if s.startswith("&"):
                s = s[1:]
            buf += " " + s
        else:
            buf = s
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        for part in _split_top(buf, ";"):
            if part.strip():
                yield part.strip()
        buf = ""


def _split_top(s: str, sep: str):
    out, depth, cur, q = [], 0, [], None
    for ch in s:
        if q:
            cur.append(ch)
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return out


# ---- expression translation ---------------------------------------------------------------------
TOK = re.compile(r"""
    (?P<ws>\s+)
  | (?P<str>'[^']*'|"[^"]*")
  | (?P<num>(\d+\.(?!(eq|ne|lt|le|gt|ge|and|or|not|eqv|neqv)\.)\d*|\.\d+|\d+)([deDE][+-]?\d+)?(_\w+)?)
  | (?P<dotop>\.(eq|ne|lt|le|gt|ge|and|or|not|true|false|eqv|neqv)\.)
  | (?P<op>\*\*|==|/=|<=|>=|=>|//|[-+*/<>(),:%=])
  | (?P<name>[a-z_][a-z0-9_]*)
""", re.X | re.I)


def tokenize(s: str):
    pos, out = 0, []
    while pos < len(s):
        m = TOK.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot tokenize {s[pos:]!r} in {s!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        val = m.group()
        if kind == "dotop":
            val = val.lower()
        elif kind == "name":
            val = val.lower()
        out.append((kind, val))
    return out


class Scope:
    """Symbol information for one procedure (arrays vs scalars vs functions)."""

    def __init__(self, arrays=(), derived=(), funcs=(), result=None):
        self.arrays = set(arrays)
        self.derived = set(derived)
        self.funcs = set(funcs)
        self.result = result


_SINGLE_LIT = re.compile(r"np\.float64\(np\.float32\(([^()]*)\)\)")


def _real_literal(txt: str) -> str:
    t = txt.lower()
    kind = None
    if "_" in t:
        t, kind = t.split("_", 1)
    if "d" in t:
        return repr(float(t.replace("d", "e"))).join(("np.float64(", ")"))
    if "." in t or "e" in t:
        if kind in ("8", "rk"):  # rk = kind(_ONE_), the double kind (register_all_variables.F90:35)
            return f"np.float64({float(t)!r})"
        # default-kind real literal: single precision, widened where used in double context
        return f"np.float64(np.float32({float(t)!r}))"
    return str(int(t))


class ExprParser:
    """Pratt parser from Fortran tokens to a Python expression string."""

    BIN = {  # op -> (precedence, right_assoc, helper)
        ".eqv.": (1, False, "_eq"), ".neqv.": (1, False, "_ne"),
        ".or.": (2, False, "_or"), ".and.": (3, False, "_and"),
        ".eq.": (5, False, "_eq"), "==": (5, False, "_eq"), ".ne.": (5, False, "_ne"), "/=": (5, False, "_ne"),
        ".lt.": (5, False, "_lt"), "<": (5, False, "_lt"), ".le.": (5, False, "_le"), "<=": (5, False, "_le"),
        ".gt.": (5, False, "_gt"), ">": (5, False, "_gt"), ".ge.": (5, False, "_ge"), ">=": (5, False, "_ge"),
        "+": (7, False, "_add"), "-": (7, False, "_sub"),
        "*": (8, False, "_mul"), "/": (8, False, "_div"),
        "**": (10, True, "_pow"),
    }

    def __init__(self, toks, scope: Scope, call_args=False):
        self.t = toks
        self.i = 0
        self.scope = scope
        self.call_args = call_args

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.t[self.i]
        if val is not None and tok[1] != val:
            raise SyntaxError(f"expected {val}, got {tok}")
        self.i += 1
        return tok

    def parse(self, minp=0):
        kind, val = self.peek()
        if val == ".not.":
            self.take()
            left = f"_not({self.parse(4)})"
        elif val in ("-", "+"):
            self.take()
            operand = self.parse(8)  # unary minus binds looser than * and /, tighter than +-
            left = f"_neg({operand})" if val == "-" else operand
        else:
            left = self.atom()
        while True:
            kind, val = self.peek()
            if val not in self.BIN:
                break
            p, right, helper = self.BIN[val]
            if p < minp:
                break
            self.take()
            rhs = self.parse(p if right else p + 1)
            # an operation between two default-kind real literals is evaluated in single precision,
            # as Fortran does (e.g. 1.0/12.0), then widened like a literal
            ml, mr = _SINGLE_LIT.fullmatch(left), _SINGLE_LIT.fullmatch(rhs)
            if ml and mr and val in ("+", "-", "*", "/"):
                a, b = np.float32(float(ml.group(1))), np.float32(float(mr.group(1)))
                with np.errstate(all="ignore"):
                    r = {"+": a + b, "-": a - b, "*": a * b, "/": a / b}[val]
                if np.isfinite(r):
                    left = f"np.float64(np.float32({float(r)!r}))"
                else:  # e.g. 0.0/0.0, the reference's way of making a NaN
                    left = f"np.float64(np.float32(float({str(float(r))!r})))"
                continue
            left = f"{helper}({left}, {rhs})"
        return left

    def atom(self):
        kind, val = self.take()
        if kind == "num":
            return _real_literal(val)
        if kind == "str":
            return repr(val[1:-1])
        if val == ".true.":
            return "True"
        if val == ".false.":
            return "False"
        if val == "(":
            e = self.parse()
            self.take(")")
            return f"({e})"
        if kind == "name":
            return self.name_ref(val)
        raise SyntaxError(f"unexpected token {val}")

    def subscripts(self):
        """Parse '(' ... ')' subscripts; returns list of (python_expr, is_section)."""
        self.take("(")
        items = []
        if self.peek()[1] == ")":
            self.take(")")
            return items
        while True:
            # keyword argument?
            if self.peek()[0] == "name" and self.peek(1)[1] == "=" and self.peek(2)[1] != "=":
                kw = self.take()[1]
                self.take("=")
                items.append((f"{kw}={self.parse()}", False))
            elif self.peek()[1] in (":",):
                self.take(":")
                hi = None if self.peek()[1] in (",", ")") else self.parse()
                items.append((f"FSlice(None, {hi})", True))
            else:
                lo = self.parse()
                if self.peek()[1] == ":":
                    self.take(":")
                    hi = None if self.peek()[1] in (",", ")") else self.parse()
                    items.append((f"FSlice({lo}, {hi})", True))
                else:
                    items.append((lo, False))
            if self.peek()[1] == ",":
                self.take(",")
                continue
            self.take(")")
            return items

    def name_ref(self, name):
        base = name
        expr = name if name not in RESERVED else name + "_"
        # component access a%b%c
        comps = []
        while self.peek()[1] == "%":
            self.take("%")
            comps.append(self.take()[1])
        if comps:
            expr = expr + "".join("." + c for c in comps)
            is_array = True
        else:
            is_array = base in self.scope.arrays
        if self.peek()[1] == "(":
            subs = self.subscripts()
            if is_array or comps:
                if any(sec for _, sec in subs):
                    return f"{expr}.section(({', '.join(e for e, _ in subs)},))" if self.call_args_ctx() else \
                        f"{expr}[{', '.join(e for e, _ in subs)}]"
                return f"{expr}[{', '.join(e for e, _ in subs)}]"
            fn = INTRINSICS.get(base, expr)
            return f"{fn}({', '.join(e for e, _ in subs)})"
        if base == self.scope.result:
            return "_result"
        return expr

    def call_args_ctx(self):
        return self.call_args


RESERVED = {"lambda", "in", "is", "not", "and", "or", "if", "else", "for", "while", "def", "class", "return",
            "pass", "from", "import", "as", "with", "global", "del", "try", "except", "raise", "yield", "print",
            "exec", "len", "id", "type", "list", "range", "min", "max", "abs", "sum", "value", "iter"}


def pyname(n: str) -> str:
    return n + "_" if n in RESERVED else n


def tr_expr(s: str, scope: Scope, call_args=False) -> str:
    p = ExprParser(tokenize(s), scope, call_args)
    e = p.parse()
    if p.i != len(p.t):
        raise SyntaxError(f"trailing tokens in {s!r}: {p.t[p.i:]}")
    return e


def tr_args(s: str, scope: Scope) -> str:
    """Translate an actual-argument list 'a, b(:,:,k), kw=c' (sections become FArr views)."""
    toks = tokenize("(" + s + ")")
    p = ExprParser(toks, scope, call_args=True)
    subs = p.subscripts()
    return ", ".join(e for e, _ in subs)


# ---- declarations ---------------------------------------------------------------------------------
TYPE_RE = re.compile(r"^(real|integer|logical|character|type\s*\(\s*\w+\s*\)|class\s*\(\s*\w+\s*\))\s*"
                     r"(\((?:[^()]|\([^()]*\))*\))?", re.I)


class Decl:
    def __init__(self, name, kind, dims=None, attrs=(), init=None, dtype_name=None):
        self.name, self.kind, self.dims, self.attrs, self.init = name, kind, dims, set(attrs), init
        self.dtype_name = dtype_name

    @property
    def is_array(self):
        return self.dims is not None


def parse_decl(stmt: str):
    m = TYPE_RE.match(stmt)
    if not m:
        return None
    tname = m.group(1).lower().replace(" ", "")
    rest = stmt[m.end():].strip()
    if tname.startswith("type(") or tname.startswith("class("):
        kind = "derived"
        dtn = tname[tname.index("(") + 1:-1]
    else:
        kind = tname
        dtn = None
    if "::" in rest:
        attr_s, ent_s = rest.split("::", 1)
        attrs = [a.strip().lower() for a in _split_top(attr_s.strip().lstrip(","), ",") if a.strip()]
    else:
        attrs, ent_s = [], rest
    dims = None
    attr_set = []
    for a in attrs:
        if a.startswith("dimension"):
            dims = a[a.index("(") + 1:a.rindex(")")]
        else:
            attr_set.append(a.split("(")[0].strip())
    out = []
    for ent in _split_top(ent_s, ","):
        ent = ent.strip()
        if not ent:
            continue
        init = None
        if "=>" in ent:
            ent, init = ent.split("=>", 1)
            init = None
        elif "=" in ent:
            ent, init = ent.split("=", 1)
        ent = ent.strip()
        ed = dims
        if "(" in ent:
            ed = ent[ent.index("(") + 1:ent.rindex(")")]
            ent = ent[:ent.index("(")].strip()
        out.append(Decl(ent.lower(), kind, ed, attr_set, init.strip() if init else None, dtn))
    return out


def dim_bounds(dims: str, scope: Scope):
    """'imin-2:imax+2, 0:kmax' -> python list-of-tuples expression; ':' -> deferred (None)."""
    parts = _split_top(dims, ",")
    out = []
    for p in parts:
        p = p.strip()
        if p in (":", "*"):
            return None
        if ":" in _top_colon(p):
            lo, hi = _split_colon(p)
            out.append(f"({tr_expr(lo, scope)}, {tr_expr(hi, scope)})")
        else:
            out.append(f"(1, {tr_expr(p, scope)})")
    return "[" + ", ".join(out) + "]"


def _top_colon(p):
    depth = 0
    for ch in p:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == ":" and depth == 0:
            return ":"
    return ""


def _split_colon(p):
    depth = 0
    for k, ch in enumerate(p):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == ":" and depth == 0:
            return p[:k], p[k + 1:]
    raise ValueError(p)


# ------------------------------------------------------------------------------------------------
# program units
class Unit:
    def __init__(self, kind, name, args=(), result=None, rtype=None):
        self.kind, self.name, self.args, self.result, self.rtype = kind, name, list(args), result, rtype
        self.uses = []  # (module, only-list or None)
        self.decls = {}
        self.body = []
        self.contains = []  # for modules


HEAD_SUB = re.compile(r"^(recursive\s+)?subroutine\s+(\w+)\s*(\((.*)\))?\s*$", re.I)
HEAD_FUN = re.compile(r"^(.*?)\bfunction\s+(\w+)\s*\((.*)\)\s*(result\s*\((\w+)\))?\s*$", re.I)
HEAD_MOD = re.compile(r"^module\s+(\w+)\s*$", re.I)


def parse_units(text: str):
    stmts = list(statements(text))
    units, i = [], 0

    def parse_proc(i, head):
        m = HEAD_SUB.match(head)
        if m:
            u = Unit("subroutine", m.group(2).lower(),
                     [a.strip().lower() for a in (m.group(4) or "").split(",") if a.strip()])
        else:
            m = HEAD_FUN.match(head)
            u = Unit("function", m.group(2).lower(), [a.strip().lower() for a in m.group(3).split(",") if a.strip()],
                     result=(m.group(5) or m.group(2)).lower(), rtype=m.group(1).strip().lower())
        i += 1
        in_body = False
        skip_depth = 0
        while i < len(stmts):
            s = stmts[i]
            low = s.lower()
            if re.match(r"^end\s*(subroutine|function)\b", low) or low == "end":
                return i + 1, u
            if skip_depth:
                if re.match(r"^end\s*(interface|type)\b", low):
                    skip_depth -= 1
                i += 1
                continue
            if re.match(r"^interface\b", low) or re.match(r"^type\s*[,:]", low) or re.match(r"^type\s+\w+\s*$", low):
                skip_depth += 1
                i += 1
                continue
            if not in_body and low.startswith("use "):
                u.uses.append(_parse_use(low))
            elif not in_body and (low.startswith("implicit") or low.startswith("private") or low.startswith("public")):
                pass
            elif not in_body and TYPE_RE.match(low) and not re.match(r"^(real|integer|logical)\s*\w*\s*function", low) \
                    and ("::" in low or re.match(r"^(real|integer|logical)(\((?:[^()]|\([^()]*\))*\)\s*|\s+)[a-z]", low)):
                for d in parse_decl(s):
                    u.decls[d.name] = d
            else:
                in_body = True
                u.body.append(s)
            i += 1
        raise SyntaxError(f"unterminated procedure {u.name}")

    while i < len(stmts):
        s = stmts[i]
        low = s.lower()
        mm = HEAD_MOD.match(low)
        if mm and not low.startswith("module procedure"):
            mod = Unit("module", mm.group(1).lower())
            i += 1
            skip_depth = 0
            while i < len(stmts):
                s2 = stmts[i]
                l2 = s2.lower()
                if re.match(r"^end\s*module\b", l2):
                    i += 1
                    break
                if skip_depth:
                    if re.match(r"^end\s*(interface|type)\b", l2):
                        skip_depth -= 1
                    i += 1
                    continue
                if re.match(r"^interface\b", l2) or re.match(r"^type\s*,", l2) or re.match(r"^type\s*::", l2) \
                        or re.match(r"^type\s+\w+\s*$", l2):
                    skip_depth += 1
                    i += 1
                    continue
                if l2 == "contains":
                    i += 1
                    continue
                if HEAD_SUB.match(l2) or (HEAD_FUN.match(l2) and re.search(r"\bfunction\s+\w+\s*\(", l2)
                                          and "::" not in l2):
                    i, u = parse_proc(i, s2)
                    mod.contains.append(u)
                    continue
                if l2.startswith("use "):
                    mod.uses.append(_parse_use(l2))
                elif TYPE_RE.match(l2):
                    for d in parse_decl(s2):
                        mod.decls[d.name] = d
                i += 1
            units.append(mod)
            continue
        if HEAD_SUB.match(low) or HEAD_FUN.match(low):
            i, u = parse_proc(i, s)
            units.append(u)
            continue
        i += 1
    return units


def _parse_use(low: str):
    m = re.match(r"^use\s+(\w+)\s*(,\s*only\s*:\s*(.*))?$", low)
    mod = m.group(1)
    only = None
    if m.group(3) is not None:
        # a renamed entity (local => remote) is listed under its local name: the module
        # namespaces this translator is given for such modules hold the local names
        only = [x.split("=>")[0].strip() for x in m.group(3).split(",") if x.strip()]
    return mod, only


# ---- code generation --------------------------------------------------------------------------------
class Gen:
    def __init__(self, unit: Unit, module_arrays=(), module_derived=(), funcs=(), modvars=()):
        self.u = unit
        self.modvars = set(modvars) - set(unit.decls) - set(unit.args) - {unit.name, unit.result}
        arrays = set(module_arrays)
        derived = set(module_derived)
        # names that the body allocates or assigns element-wise are arrays even when their
        # declaration lives in a module this translator has only as a namespace
        for s in unit.body:
            low = s.lower()
            m = re.match(r"^allocate\s*\((.*)\)$", low)
            if m:
                for item in _split_top(m.group(1), ","):
                    item = item.strip()
                    if "(" in item and "%" not in item.split("(")[0]:
                        arrays.add(item[:item.index("(")].strip())
                continue
            m = re.match(r"^(\w+)\s*\(", low)
            if m and m.group(1) not in ("if", "call", "do", "select", "case", "allocate", "deallocate", "write",
                                        "print", "where", "elseif") and _top_assign(low) is not None:
                arrays.add(m.group(1))
        for d in unit.decls.values():
            if d.is_array:
                arrays.add(d.name)
            if d.kind == "derived":
                derived.add(d.name)
        self.scope = Scope(arrays, derived, funcs, unit.result if unit.kind == "function" else None)
        self.lines = []
        self.ind = 1
        self.sel = 0
        self.saved = []

    def emit(self, s):
        if self.lines and self.lines[-1].rstrip().endswith(":"):
            prev = self.lines[-1]
            prev_ind = len(prev) - len(prev.lstrip(" "))
            if 4 * self.ind <= prev_ind:  # empty block (e.g. 'case (2) ! z-level')
                self.lines.append(" " * (prev_ind + 4) + "pass")
        self.lines.append("    " * self.ind + s)

    def gen(self) -> str:
        u = self.u
        args = []
        for a in u.args:
            d = u.decls.get(a)
            opt = d is not None and "optional" in d.attrs
            args.append(f"{pyname(a)}=None" if opt else pyname(a))
        # Python requires non-defaults first: all optionals in the reference come last
        self.lines.append(f"def {u.name}({', '.join(args)}):")
        assigned = self._assigned_names()
        self.assigned_globals = sorted(assigned & self.modvars)
        if self.assigned_globals:
            self.emit(f"global {', '.join(pyname(n) for n in self.assigned_globals)}")
        self.emit("_result = None")
        # a subroutine hands the final values of the scalar dummies it assigns back to its caller
        outs = [(q, a) for q, a in enumerate(u.args)
                if u.kind != "function" and a in assigned and not (u.decls.get(a) is not None and u.decls[a].is_array)]
        self.ret = "_result"
        if outs:
            self.emit("_ret = lambda: _Out({" + ", ".join(f"{q}: {pyname(a)}" for q, a in outs) + "})")
            self.ret = "_ret()"
        # parameters and locals (in declaration order, so that bounds can use earlier ones)
        for name, d in u.decls.items():
            if name == u.result and u.kind == "function":
                continue
            kind = "real" if d.kind.startswith("real") else d.kind
            if name in u.args:
                if d.is_array and d.dims is not None:
                    b = dim_bounds(d.dims, self.scope)
                    if b is not None:
                        self.emit(f"{pyname(name)} = _bind({pyname(name)}, {b}, {kind!r})")
                continue
            if "parameter" in d.attrs:
                self.emit(f"{pyname(name)} = {tr_expr(d.init, self.scope)}")
                continue
            if d.kind == "derived":
                self.emit(f"{pyname(name)} = None")
                continue
            saved = "save" in d.attrs or d.init is not None  # explicit SAVE or implicit (initialiser)
            if saved:
                self.saved.append(name)
            if d.is_array:
                b = dim_bounds(d.dims, self.scope)
                if b is None or "allocatable" in d.attrs or "pointer" in d.attrs:
                    init = "None"
                else:
                    init = f"_alloc({b}, {kind!r})"
            else:
                init = tr_expr(d.init, self.scope) if d.init else {"real": "np.float64(0)", "integer": "0",
                                                                   "logical": "False"}.get(kind, "None")
            if saved:
                self.emit(f"{pyname(name)} = _SV[{name!r}] if {name!r} in _SV else {init}")
            else:
                self.emit(f"{pyname(name)} = {init}")
        if self.saved:
            # SAVEd locals persist across calls (written back on every exit)
            self.emit("try:")
            self.ind += 1
        for s in u.body:
            self.stmt(s)
        self.emit(f"return {self.ret}")
        if self.saved:
            self.ind -= 1
            self.emit("finally:")
            self.ind += 1
            for name in self.saved:
                self.emit(f"_SV[{name!r}] = {pyname(name)}")
            self.ind -= 1
        return "\n".join(self.lines)

    def stmt(self, s: str):
        low = s.lower().strip()
        sc = self.scope
        # WHERE constructs (block and single-statement forms) with plain array assignments
        if not hasattr(self, "wstack"):
            self.wstack, self.nwhere = [], 0
        m = re.match(r"^where\s*\((.*)$", low)
        if m and not low.startswith("where_"):
            rest = low[low.index("("):]
            depth, q = 0, 0
            for q, ch in enumerate(rest):
                depth += ch == "("
                depth -= ch == ")"
                if depth == 0:
                    break
            cond, tail = rest[1:q], rest[q + 1:].strip()
            self.nwhere += 1
            w = f"_w{self.nwhere}"
            self.emit(f"{w} = np.asarray(_arr({tr_expr(cond, sc)}), dtype=bool)")
            self.wstack.append(w)
            if tail:
                self.stmt(tail)
                self.wstack.pop()
            return
        if re.match(r"^else\s*where$", low):
            w = self.wstack[-1]
            self.emit(f"{w} = ~{w}")
            return
        if re.match(r"^end\s*where$", low):
            self.wstack.pop()
            return
        if self.wstack:
            k = _top_assign(low)
            if k is None:
                raise SyntaxError(f"unsupported statement in WHERE: {s}")
            lhs = low[:k].strip()
            if not re.match(r"^\w+$", lhs):
                raise SyntaxError(f"unsupported WHERE assignment target: {s}")
            self.emit(f"_wassign({pyname(lhs)}, {tr_expr(low[k + 1:].strip(), sc)}, {self.wstack[-1]})")
            return
        m = re.match(r"^if\s*\((.*)\)\s*then$", low)
        if m and _balanced_prefix(low[2:].strip()):
            self.emit(f"if {tr_expr(m.group(1), sc)}:")
            self.ind += 1
            return
        m = re.match(r"^else\s*if\s*\((.*)\)\s*then$", low)
        if m:
            self.ind -= 1
            self.emit(f"elif {tr_expr(m.group(1), sc)}:")
            self.ind += 1
            return
        if low == "else":
            self.ind -= 1
            self.emit("else:")
            self.ind += 1
            return
        if re.match(r"^end\s*if$", low):
            self.emit("pass")
            self.ind -= 1
            return
        if low.startswith("if") and re.match(r"^if\s*\(", low):
            cond, rest = _split_if(low)
            self.emit(f"if {tr_expr(cond, sc)}:")
            self.ind += 1
            self.stmt(rest)
            self.ind -= 1
            return
        if low == "do":  # a DO without control, left by EXIT
            self.emit("while True:")
            self.ind += 1
            return
        m = re.match(r"^do\s+while\s*\((.*)\)$", low)
        if m:
            self.emit(f"while {tr_expr(m.group(1), sc)}:")
            self.ind += 1
            return
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", low)
        if m:
            parts = _split_top(m.group(2), ",")
            rng = ", ".join(tr_expr(p, sc) for p in parts)
            self.emit(f"for {m.group(1)} in _range({rng}):")
            self.ind += 1
            return
        if re.match(r"^end\s*do$", low):
            self.emit("pass")
            self.ind -= 1
            return
        m = re.match(r"^select\s+case\s*\((.*)\)$", low)
        if m:
            self.sel += 1
            self.emit(f"_sel{self.sel} = {tr_expr(m.group(1), sc)}")
            self.emit("if False:")
            self.ind += 1
            self.emit("pass")
            return
        m = re.match(r"^case\s*\((.*)\)$", low)
        if m:
            vals = [tr_expr(v.strip().strip("()") if v.strip().startswith("(") and v.strip().endswith(")") else v, sc)
                    for v in _split_top(m.group(1), ",")]
            self.ind -= 1
            self.emit(f"elif _sel{self.sel} in ({', '.join(vals)},):")
            self.ind += 1
            return
        if re.match(r"^case\s+default$", low):
            self.ind -= 1
            self.emit("else:")
            self.ind += 1
            return
        if re.match(r"^end\s*select$", low):
            self.emit("pass")
            self.ind -= 1
            self.sel -= 1
            return
        if low == "return":
            self.emit(f"return {self.ret}")
            return
        if low == "cycle":
            self.emit("continue")
            return
        if low == "exit":
            self.emit("break")
            return
        if low.startswith("stop"):
            self.emit(f"raise FortranStop({low[4:].strip()!r})")
            return
        if low.startswith("write") or low.startswith("print"):
            self.emit("_write()")
            return
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", low)
        if m:
            name = m.group(1)
            args = tr_args(m.group(3), sc) if m.group(3) else ""
            # actual arguments that a scalar out-argument can be copied back into: plain local or
            # module-assigned variables and array elements, by position (keyword arguments excluded)
            back = []
            if m.group(3):
                for q, a in enumerate(_split_top(m.group(3), ",")):
                    a = a.strip()
                    if _top_assign(a) is not None:
                        break
                    d = self.u.decls.get(a)
                    if d is not None and "parameter" in d.attrs:
                        continue
                    if re.match(r"^[a-z_]\w*$", a) and a not in self.u.args and (a not in self.modvars or
                                                                                 a in self.assigned_globals):
                        if d is None or not d.is_array:
                            back.append((q, pyname(a)))
                    elif re.match(r"^\w+\s*\(.*\)$", a) and a[:a.index("(")].strip() in self.scope.arrays:
                        back.append((q, tr_expr(a, sc)))
                    elif re.match(r"^[a-z_]\w*$", a) and a in self.u.args:
                        if d is not None and not d.is_array:
                            back.append((q, pyname(a)))
            if back:
                self.emit(f"_r = {name}({args})")
                self.emit("if isinstance(_r, _Out):")
                self.ind += 1
                for q, tgt in back:
                    self.emit(f"if {q} in _r: {tgt} = _r[{q}]")
                self.ind -= 1
            else:
                self.emit(f"{name}({args})")
            return
        m = re.match(r"^allocate\s*\((.*)\)$", low)
        if m:
            for item in _split_top(m.group(1), ","):
                item = item.strip()
                if item.startswith("stat"):
                    var = item.split("=", 1)[1].strip()
                    self.emit(f"{var} = 0")
                    continue
                nm = item[:item.index("(")].strip()
                dims = item[item.index("(") + 1:item.rindex(")")]
                kind = self._kind_of(nm)
                target = tr_expr(nm, sc) if "%" in nm else nm
                self.emit(f"{target} = _alloc({dim_bounds(dims, sc)}, {kind!r})")
            return
        m = re.match(r"^deallocate\s*\((.*)\)$", low)
        if m:
            for item in _split_top(m.group(1), ","):
                if item.strip().startswith("stat"):
                    self.emit(f"{item.split('=', 1)[1].strip()} = 0")
            return
        if "=>" in low and _top_arrow(low):
            lhs, rhs = low.split("=>", 1)
            self.emit(f"{self._lhs_target(lhs.strip())} = {tr_expr(rhs.strip(), sc, call_args=True)}")
            return
        # assignment
        k = _top_assign(low)
        if k is not None:
            lhs, rhs = low[:k].strip(), low[k + 1:].strip()
            r = tr_expr(rhs, sc)
            base = re.match(r"^(\w+)", lhs).group(1)
            if self.u.kind == "function" and base == self.u.result and "(" not in lhs:
                self.emit(f"_result = {r}")
                return
            if "(" in lhs or "%" in lhs:
                tgt = tr_expr(lhs, sc)
                if "%" in lhs and "(" not in lhs.split("%")[-1]:
                    self.emit(f"_assign({tgt}, {r}) if isinstance({tgt}, FArr) else None")
                    if not self._comp_is_array(lhs):
                        self.lines.pop()
                        self.emit(f"{tgt} = {r}")
                else:
                    self.emit(f"{tgt} = {r}")
                return
            if base in sc.arrays:
                self.emit(f"_assign({pyname(lhs)}, {r})")
            else:
                self.emit(f"{lhs if lhs not in RESERVED else lhs + '_'} = {r}")
            return
        raise SyntaxError(f"unsupported statement: {s}")

    def _assigned_names(self):
        """Bare names that the body (re)binds: scalar assignment, allocate, pointer assignment."""
        out = set()
        for s in self.u.body:
            low = s.lower().strip()
            m = re.match(r"^if\s*\(", low)
            if m and not low.endswith("then"):
                try:
                    low = _split_if(low)[1]
                except SyntaxError:
                    pass
            m = re.match(r"^allocate\s*\((.*)\)$", low)
            if m:
                for item in _split_top(m.group(1), ","):
                    item = item.strip()
                    if "(" in item and "%" not in item.split("(")[0]:
                        out.add(item[:item.index("(")].strip())
                continue
            if "=>" in low and _top_arrow(low):
                lhs = low.split("=>", 1)[0].strip()
                if re.match(r"^\w+$", lhs):
                    out.add(lhs)
                continue
            k = _top_assign(low)
            if k is not None and not re.match(r"^(do|if|else|select|case|call)\b", low):
                lhs = low[:k].strip()
                if re.match(r"^\w+$", lhs):
                    out.add(lhs)
        return out

    def _kind_of(self, nm):
        d = self.u.decls.get(nm.split("%")[0])
        if d is None:
            return "real"
        return "real" if d.kind.startswith("real") else d.kind

    def _comp_is_array(self, lhs):
        return True

    def _lhs_target(self, lhs):
        # pointer (re)association target: plain name or component
        if "(" in lhs:
            lhs = lhs[:lhs.index("(")]
        return tr_expr(lhs, self.scope)


def _balanced_prefix(s):
    # 'if (...) then' where the parenthesis closes right before 'then'
    depth = 0
    for k, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
            if depth == 0:
                return s[k + 1:].strip() == "then"
    return False


def _split_if(low):
    depth = 0
    start = low.index("(")
    for k in range(start, len(low)):
        if low[k] == "(":
            depth += 1
        elif low[k] == ")":
            depth -= 1
            if depth == 0:
                return low[start + 1:k], low[k + 1:].strip()
    raise SyntaxError(low)


def _top_assign(s):
    depth, q = 0, None
    for k, ch in enumerate(s):
        if q:
            if ch == q:
                q = None
            continue
        if ch in "'\"":
            q = ch
        elif ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            prev = s[k - 1] if k else ""
            nxt = s[k + 1] if k + 1 < len(s) else ""
            if prev in "<>/=" or nxt in "=>":
                continue
            return k
    return None


def _top_arrow(s):
    depth = 0
    for k, ch in enumerate(s):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0 and k + 1 < len(s) and s[k + 1] == ">":
            return True
    return False


# ------------------------------------------------------------------------------------------------
class Program:
    """A set of translated reference files sharing module namespaces."""

    def __init__(self, defines=()):
        self.defines = defines
        self.modules = {}     # name -> types.SimpleNamespace of module variables/procedures
        self.mod_units = {}
        self.procs = {}       # external procedures
        self.sources = {}

    def visible(self, mname, _seen=None):
        """Names a `use mname` makes visible: the module's own entities and, transitively, those of
        the modules it uses (use-association re-exports them unless private)."""
        seen = _seen if _seen is not None else set()
        if mname in seen:
            return {}
        seen.add(mname)
        out = {}
        mu = self.mod_units.get(mname)
        if mu is not None:
            for sub, only in mu.uses:
                for k, v in self.visible(sub, set(seen)).items():
                    if only is None or k in only:
                        out[k] = v
        mns = self.modules.get(mname)
        if mns is not None:
            out.update(vars(mns))
        return out

    def visible_owner(self, mname, _seen=None):
        """Like visible(), mapping each name to the module whose namespace holds it."""
        seen = _seen if _seen is not None else set()
        if mname in seen:
            return {}
        seen.add(mname)
        out = {}
        mu = self.mod_units.get(mname)
        if mu is not None:
            for sub, only in mu.uses:
                for k, o in self.visible_owner(sub, set(seen)).items():
                    if only is None or k in only:
                        out[k] = o
            for k in mu.decls:
                out[k] = mname
        mns = self.modules.get(mname)
        if mns is not None:
            for k in vars(mns):
                out[k] = mname
        return out

    def add_module_namespace(self, name, **values):
        ns = self.modules.setdefault(name, types.SimpleNamespace())
        for k, v in values.items():
            setattr(ns, k.lower(), v)
        return ns

    def load(self, relpath: str):
        path = os.path.join(REF, relpath)
        units = parse_units(preprocess(path, self.defines))
        for u in units:
            if u.kind == "module":
                self.mod_units[u.name] = u
                ns = self.modules.setdefault(u.name, types.SimpleNamespace())
                # module parameters and variables
                for d in u.decls.values():
                    if "parameter" in d.attrs and d.init is not None:
                        if d.dims is not None:
                            continue  # character parameter arrays (names of schemes)
                        try:
                            val = eval(tr_expr(d.init, Scope()), self._globals(u, ns))
                        except Exception:
                            continue
                        setattr(ns, d.name, val)
                    elif d.kind == "derived":
                        if not hasattr(ns, d.name):
                            setattr(ns, d.name, types.SimpleNamespace())
                    elif not hasattr(ns, d.name):
                        setattr(ns, d.name, None if d.is_array else (False if d.kind == "logical" else 0))
                for p in u.contains:
                    self._compile(p, u, ns)
            else:
                self._compile(u, None, None)
        return self

    def _module_arrays(self, unit: Unit, mod: Unit | None):
        arrays, derived = set(), set()
        sources = []
        if mod is not None:
            sources.append((mod, None))
        for mname, only in unit.uses + (mod.uses if mod else []):
            mu = self.mod_units.get(mname)
            if mu is not None:
                sources.append((mu, only))
            for k, v in self.visible(mname).items():
                if only is None or k in only:
                    declared_array = any(m.decls.get(k) is not None and m.decls[k].is_array
                                         for m in self.mod_units.values())
                    if isinstance(v, FArr) or (v is None and declared_array):
                        arrays.add(k)
                    if isinstance(v, types.SimpleNamespace):
                        derived.add(k)
        for mu, only in sources:
            for k, d in mu.decls.items():
                if only is None or k in only:
                    if d.is_array:
                        arrays.add(k)
                    if d.kind == "derived":
                        derived.add(k)
        return arrays, derived

    def _globals(self, unit: Unit | None, ns):
        g = {k: v for k, v in globals().items() if k.startswith("_") or k in ("np", "FArr", "FSlice", "FortranStop")}
        return g

    def _compile(self, unit: Unit, mod: Unit | None, ns):
        prog = self
        modname = mod.name if mod else None
        saved_store = {}  # SAVEd locals of this procedure
        cache = {}

        def translate():
            # translated on first call, once every file of the program is loaded
            arrays, derived = prog._module_arrays(unit, mod)
            owner = {}
            uses = ([(mod.name, None)] + list(mod.uses) if mod else []) + list(unit.uses)
            for mname, only in uses:
                for k, o in prog.visible_owner(mname).items():
                    if only is None or k in only:
                        owner.setdefault(k, o)
            for k, d in unit.decls.items():  # names declared locally shadow module arrays
                if not d.is_array and k in arrays:
                    arrays.discard(k)
            gen = Gen(unit, arrays, derived, modvars=owner.keys())
            try:
                src = gen.gen()
            except SyntaxError as ex:
                # routines outside the supported subset (namelist / netCDF I/O, ...) fail only if called
                raise NotImplementedError(f"{unit.name}: not translatable ({ex})")
            prog.sources[unit.name] = src
            cache.update(src=src, gen=gen, owner=owner, code=compile(src, f"<{unit.name}>", "exec"))

        def runner(*args, **kw):
            if not cache:
                translate()
            gen, owner = cache["gen"], cache["owner"]
            g = prog._globals(unit, ns)
            # resolve module names at call time (use-association)
            uses = list(unit.uses)
            if mod is not None:
                uses = [(mod.name, None)] + list(mod.uses) + uses
            for mname, only in uses:
                for k, v in prog.visible(mname).items():
                    if only is None or k in only:
                        g[k] = v
            for k, v in prog.procs.items():
                g.setdefault(k, v)
            if modname:
                for k, v in vars(prog.modules[modname]).items():
                    g.setdefault(k, v)
            g["_SV"] = saved_store
            loc = {}
            exec(cache["code"], g, loc)
            fn = loc[unit.name]
            try:
                return fn(*args, **kw)
            finally:
                for n in gen.assigned_globals:
                    if pyname(n) in g:
                        setattr(prog.modules.setdefault(owner[n], types.SimpleNamespace()), n, g[pyname(n)])

        runner.__name__ = unit.name
        if mod is not None:
            setattr(ns, unit.name, runner)
        self.procs[unit.name] = runner
