"""mlite - a MATLAB-subset interpreter used to run SCMC's own .m files.

Neither MATLAB nor GNU Octave is available to this build, and the reference
(cmu-ci-lab/mcspeckle) stores no output vectors.  To pin the CPU oracle to
the reference itself, this interpreter executes the reference's .m sources
unmodified (code/MCfield.m, code/MCcov.m, code/MCfieldFourierQuad.m, the
coreFunctions they call and the interface/ constructors) with `rand` and
`randn` served from recorded tapes.  The outputs become the golden fixtures
in tests/golden/.

It implements the part of the language those files use: numeric / logical /
complex N-d arrays with MATLAB's column-major indexing, growth on assignment,
`end` in subscripts, implicit expansion, 1x1 structs, cells for varargin,
if / elseif / else, for / parfor, while, switch, break / continue / return,
multiple return values, and the builtins listed in BUILTINS.  MATLAB's
automatic complex results (sqrt / log / acos / power of out-of-domain reals),
round-half-away-from-zero and short-circuit `&` / `|` in if / while
conditions are reproduced.  It is test tooling: it never ships and never runs
on the GPU box.
"""
from __future__ import annotations

import math
import os
import re

import numpy as np


class MatlabError(Exception):
    """An error() raised by the interpreted code (message kept verbatim)."""


class _Break(Exception):
    pass


class _Continue(Exception):
    pass


class _Return(Exception):
    pass


# ----------------------------------------------------------------------------
# values
# ----------------------------------------------------------------------------

class MStruct(dict):
    pass


class MCell:
    def __init__(self, items):
        self.items = list(items)


class FHandle:
    def __init__(self, name):
        self.name = name


class MStr(str):
    """A MATLAB char row vector."""


def M(x):
    """Python / numpy value -> MATLAB array (ndim >= 2)."""
    if isinstance(x, (MStr, MStruct, MCell, FHandle)):
        return x
    if isinstance(x, str):
        return MStr(x)
    a = np.asarray(x)
    if a.dtype == object:
        raise TypeError("object array")
    if a.ndim == 0:
        a = a.reshape(1, 1)
    elif a.ndim == 1:
        a = a.reshape(1, -1)
    return _squeeze_trailing(a)


def _squeeze_trailing(a):
    while a.ndim > 2 and a.shape[-1] == 1:
        a = a.reshape(a.shape[:-1])
    return a


def _realify(a):
    if isinstance(a, np.ndarray) and np.iscomplexobj(a) and a.size and not np.any(a.imag):
        return a.real.copy()
    return a


def num(a):
    """MATLAB array -> numeric numpy array (char arrays become codes)."""
    if isinstance(a, MStr):
        return np.array([[ord(c) for c in a]], dtype=float).reshape(1, len(a))
    if isinstance(a, np.ndarray):
        return a
    return M(a)


def scalar(a):
    a = num(a)
    if a.size != 1:
        raise MatlabError("expected a scalar")
    v = a.reshape(-1)[0]
    return v.item() if hasattr(v, "item") else v


def truth(a):
    if isinstance(a, MStr):
        return len(a) > 0 and all(ord(c) != 0 for c in a)
    a = num(a)
    if a.size == 0:
        return False
    if np.iscomplexobj(a):
        a = a.real
    return bool(np.all(a != 0))


def _as_float(a):
    a = num(a)
    if a.dtype == bool or np.issubdtype(a.dtype, np.integer):
        return a.astype(float)
    return a


# ----------------------------------------------------------------------------
# lexer
# ----------------------------------------------------------------------------

KEYWORDS = {"function", "end", "if", "elseif", "else", "for", "parfor", "while", "switch",
            "case", "otherwise", "break", "continue", "return", "global", "persistent"}

_OPS = ["...", ".^", ".*", "./", ".\\", ".'", "==", "~=", "<=", ">=", "&&", "||",
        "+", "-", "*", "/", "\\", "^", "<", ">", "&", "|", "~", "!", "=", ":", ",", ";",
        "(", ")", "[", "]", "{", "}", ".", "@", "'"]

_NUM_RE = re.compile(r"(\d+(?:\.(?![*/\\^'])\d*)?|\.\d+)([eE][+-]?\d+)?([ij](?![A-Za-z0-9_]))?")
_ID_RE = re.compile(r"[A-Za-z_][A-Za-z0-9_]*")


class Tok:
    __slots__ = ("kind", "val", "line")

    def __init__(self, kind, val, line):
        self.kind, self.val, self.line = kind, val, line

    def __repr__(self):
        return f"{self.kind}:{self.val!r}@{self.line}"


def lex(src):
    toks = []
    i, n, line = 0, len(src), 1
    stack = []  # bracket stack: '(', '[', '{'

    def prev_is_value():
        if not toks:
            return False
        t = toks[-1]
        if t.kind in ("num", "id", "str"):
            return True
        if t.kind == "kw" and t.val == "end":
            return True
        return t.kind == "op" and t.val in (")", "]", "}", "'", ".'")

    while i < n:
        c = src[i]
        ws = False
        while i < n and src[i] in " \t\r":
            i += 1
            ws = True
        if i >= n:
            break
        c = src[i]
        in_mat = bool(stack) and stack[-1] in "[{"
        if c == "%":
            while i < n and src[i] != "\n":
                i += 1
            continue
        if src.startswith("...", i):
            while i < n and src[i] != "\n":
                i += 1
            i += 1
            line += 1
            continue
        if c == "\n":
            line += 1
            i += 1
            if in_mat:
                toks.append(Tok("op", ";", line))
            elif not stack:
                toks.append(Tok("nl", "\n", line))
            continue
        # whitespace separating matrix elements
        if in_mat and ws and prev_is_value():
            starts_value = (c.isalnum() or c in "_.([{@'\"" or (c == "~" and src[i + 1:i + 2] != "="))
            if c in "+-" and i + 1 < n and src[i + 1] not in " \t":
                starts_value = True
            if c == "." and not (i + 1 < n and src[i + 1].isdigit()):
                starts_value = False
            if starts_value:
                toks.append(Tok("op", ",", line))
        if c == "'":
            if prev_is_value() and not (in_mat and ws):
                toks.append(Tok("op", "'", line))
                i += 1
                continue
            j = i + 1
            buf = []
            while j < n:
                if src[j] == "'":
                    if j + 1 < n and src[j + 1] == "'":
                        buf.append("'")
                        j += 2
                        continue
                    break
                buf.append(src[j])
                j += 1
            toks.append(Tok("str", "".join(buf), line))
            i = j + 1
            continue
        if c == '"':
            j = i + 1
            buf = []
            while j < n and src[j] != '"':
                buf.append(src[j])
                j += 1
            toks.append(Tok("str", "".join(buf), line))
            i = j + 1
            continue
        if c.isdigit() or (c == "." and i + 1 < n and src[i + 1].isdigit()):
            m = _NUM_RE.match(src, i)
            text = m.group(1) + (m.group(2) or "")
            val = float(text)
            if m.group(3):
                toks.append(Tok("num", complex(0.0, val), line))
            else:
                toks.append(Tok("num", val, line))
            i = m.end()
            continue
        if c.isalpha() or c == "_":
            m = _ID_RE.match(src, i)
            w = m.group(0)
            after_dot = bool(toks) and toks[-1].kind == "op" and toks[-1].val == "."
            toks.append(Tok("kw" if (w in KEYWORDS and not after_dot) else "id", w, line))
            i = m.end()
            continue
        for op in _OPS:
            if src.startswith(op, i):
                if op == ".'" and not prev_is_value():
                    continue
                if op in ("(", "[", "{"):
                    stack.append(op)
                elif op in (")", "]", "}"):
                    if stack:
                        stack.pop()
                if op == "," and not stack:
                    toks.append(Tok("nl", ",", line))
                elif op == ";" and not stack:
                    toks.append(Tok("nl", ";", line))
                else:
                    toks.append(Tok("op", op, line))
                i += len(op)
                break
        else:
            raise SyntaxError(f"unexpected character {c!r} at line {line}")
    toks.append(Tok("eof", None, line))
    return toks


# ----------------------------------------------------------------------------
# parser (AST as tuples)
# ----------------------------------------------------------------------------

class Parser:
    def __init__(self, toks):
        self.t = toks
        self.p = 0
        self.index_depth = 0

    def peek(self, k=0):
        return self.t[self.p + k]

    def next(self):
        tok = self.t[self.p]
        self.p += 1
        return tok

    def accept(self, kind, val=None):
        tok = self.peek()
        if tok.kind == kind and (val is None or tok.val == val):
            self.p += 1
            return tok
        return None

    def expect(self, kind, val=None):
        tok = self.accept(kind, val)
        if tok is None:
            raise SyntaxError(f"expected {kind} {val!r}, got {self.peek()!r}")
        return tok

    def skip_nl(self):
        while self.peek().kind == "nl":
            self.p += 1

    # -- file -------------------------------------------------------------
    def parse_file(self):
        funcs = {}
        order = []
        self.skip_nl()
        while self.peek().kind != "eof":
            if self.peek().kind == "kw" and self.peek().val == "function":
                f = self.parse_function()
                funcs[f["name"]] = f
                order.append(f["name"])
            else:
                raise SyntaxError(f"script files are not supported ({self.peek()!r})")
            self.skip_nl()
        return funcs, order

    def parse_function(self):
        self.expect("kw", "function")
        outs = []
        # forms: function name(...), function out = name(...), function [a,b] = name(...)
        if self.accept("op", "["):
            while not self.accept("op", "]"):
                tok = self.next()
                if tok.kind == "id":
                    outs.append(tok.val)
            self.expect("op", "=")
            name = self.expect("id").val
        else:
            first = self.expect("id").val
            if self.accept("op", "="):
                outs = [first]
                name = self.expect("id").val
            else:
                name = first
        params = []
        if self.accept("op", "("):
            while not self.accept("op", ")"):
                tok = self.next()
                if tok.kind == "id":
                    params.append(tok.val)
                elif tok.kind == "op" and tok.val == "~":
                    params.append("~")
        body = self.parse_block(("function",), top=True)
        if self.peek().kind == "kw" and self.peek().val == "end":
            self.next()
        return {"name": name, "outs": outs, "params": params, "body": body}

    def parse_block(self, terminators, top=False):
        stmts = []
        while True:
            self.skip_nl()
            tok = self.peek()
            if tok.kind == "eof":
                return stmts
            if tok.kind == "kw" and (tok.val in terminators or tok.val in ("end", "elseif", "else", "case", "otherwise")):
                return stmts
            stmts.append(self.parse_stmt())

    def parse_stmt(self):
        tok = self.peek()
        if tok.kind == "kw":
            kw = tok.val
            if kw == "if":
                self.next()
                clauses = []
                cond = self.parse_expr()
                body = self.parse_block(())
                clauses.append((cond, body))
                els = None
                while True:
                    t = self.next()
                    if t.val == "elseif":
                        cond = self.parse_expr()
                        body = self.parse_block(())
                        clauses.append((cond, body))
                    elif t.val == "else":
                        els = self.parse_block(())
                    elif t.val == "end":
                        break
                    else:
                        raise SyntaxError(f"bad if at {t!r}")
                return ("if", clauses, els)
            if kw in ("for", "parfor"):
                self.next()
                paren = self.accept("op", "(")
                var = self.expect("id").val
                self.expect("op", "=")
                rng = self.parse_expr()
                if paren:
                    self.expect("op", ")")
                body = self.parse_block(())
                self.expect("kw", "end")
                return ("for", var, rng, body)
            if kw == "while":
                self.next()
                cond = self.parse_expr()
                body = self.parse_block(())
                self.expect("kw", "end")
                return ("while", cond, body)
            if kw == "switch":
                self.next()
                subj = self.parse_expr()
                cases = []
                other = None
                self.skip_nl()
                while True:
                    self.skip_nl()
                    t = self.next()
                    if t.val == "case":
                        val = self.parse_expr()
                        body = self.parse_block(())
                        cases.append((val, body))
                    elif t.val == "otherwise":
                        other = self.parse_block(())
                    elif t.val == "end":
                        break
                    else:
                        raise SyntaxError(f"bad switch at {t!r}")
                return ("switch", subj, cases, other)
            if kw in ("break", "continue", "return"):
                self.next()
                return (kw,)
            if kw in ("global", "persistent"):
                raise SyntaxError(f"{kw} not supported")
        # multi-assignment [a, b] = ...
        if tok.kind == "op" and tok.val == "[" and self._is_multi_assign():
            self.next()
            targets = []
            while True:
                if self.accept("op", "]"):
                    break
                if self.accept("op", ","):
                    continue
                if self.peek().kind == "op" and self.peek().val == "~":
                    self.next()
                    targets.append(None)
                    continue
                targets.append(self.parse_postfix())
            self.expect("op", "=")
            rhs = self.parse_expr()
            return ("massign", targets, rhs)
        e = self.parse_expr()
        if self.accept("op", "="):
            rhs = self.parse_expr()
            return ("assign", e, rhs)
        return ("expr", e)

    def _is_multi_assign(self):
        depth = 0
        k = self.p
        while True:
            t = self.t[k]
            if t.kind == "eof" or t.kind == "nl":
                return False
            if t.kind == "op" and t.val in "([{":
                depth += 1
            elif t.kind == "op" and t.val in ")]}":
                depth -= 1
                if depth == 0:
                    nt = self.t[k + 1]
                    return nt.kind == "op" and nt.val == "="
            k += 1

    # -- expressions ------------------------------------------------------
    def parse_expr(self):
        return self.parse_oror()

    def _binary(self, sub, ops):
        left = sub()
        while self.peek().kind == "op" and self.peek().val in ops:
            op = self.next().val
            right = sub()
            left = ("bin", op, left, right)
        return left

    def parse_oror(self):
        return self._binary(self.parse_andand, ("||",))

    def parse_andand(self):
        return self._binary(self.parse_or, ("&&",))

    def parse_or(self):
        return self._binary(self.parse_and, ("|",))

    def parse_and(self):
        return self._binary(self.parse_cmp, ("&",))

    def parse_cmp(self):
        return self._binary(self.parse_range, ("==", "~=", "<", "<=", ">", ">="))

    def parse_range(self):
        if self.index_depth and self.peek().kind == "op" and self.peek().val == ":":
            nt = self.peek(1)
            if nt.kind == "op" and nt.val in (",", ")", "}"):
                self.next()
                return ("colon_all",)
        a = self.parse_add()
        if self.peek().kind == "op" and self.peek().val == ":":
            self.next()
            b = self.parse_add()
            if self.peek().kind == "op" and self.peek().val == ":":
                self.next()
                c = self.parse_add()
                return ("range", a, b, c)
            return ("range", a, None, b)
        return a

    def parse_add(self):
        return self._binary(self.parse_mul, ("+", "-"))

    def parse_mul(self):
        return self._binary(self.parse_unary, ("*", "/", ".*", "./", "\\", ".\\"))

    def parse_unary(self):
        t = self.peek()
        if t.kind == "op" and t.val in ("-", "+", "~", "!"):
            self.next()
            operand = self.parse_unary()
            return ("un", "~" if t.val == "!" else t.val, operand)
        return self.parse_power()

    def parse_power(self):
        left = self.parse_postfix()
        while self.peek().kind == "op" and self.peek().val in ("^", ".^"):
            op = self.next().val
            right = self.parse_power_operand()
            left = ("bin", op, left, right)
        return left

    def parse_power_operand(self):
        t = self.peek()
        if t.kind == "op" and t.val in ("-", "+", "~", "!"):
            self.next()
            return ("un", "~" if t.val == "!" else t.val, self.parse_power_operand())
        return self.parse_postfix()

    def parse_args(self, close):
        args = []
        self.index_depth += 1
        try:
            if self.accept("op", close):
                return args
            while True:
                args.append(self.parse_expr())
                if self.accept("op", close):
                    return args
                self.expect("op", ",")
        finally:
            self.index_depth -= 1

    def parse_postfix(self):
        e = self.parse_primary()
        while True:
            t = self.peek()
            if t.kind != "op":
                break
            if t.val == "(":
                self.next()
                e = ("call", e, self.parse_args(")"))
            elif t.val == "{":
                self.next()
                e = ("cellidx", e, self.parse_args("}"))
            elif t.val == "." and self.peek(1).kind == "id":
                self.next()
                e = ("field", e, self.next().val)
            elif t.val == "'":
                self.next()
                e = ("ctranspose", e)
            elif t.val == ".'":
                self.next()
                e = ("transpose", e)
            else:
                break
        return e

    def parse_primary(self):
        t = self.next()
        if t.kind == "num":
            return ("num", t.val)
        if t.kind == "str":
            return ("str", t.val)
        if t.kind == "id":
            return ("id", t.val)
        if t.kind == "kw" and t.val == "end" and self.index_depth:
            return ("end",)
        if t.kind == "op":
            if t.val == "(":
                saved = self.index_depth
                self.index_depth = 0
                e = self.parse_expr()
                self.index_depth = saved
                self.expect("op", ")")
                return ("paren", e)
            if t.val in ("[", "{"):
                close = "]" if t.val == "[" else "}"
                saved = self.index_depth
                self.index_depth = 0
                rows = [[]]
                while True:
                    if self.accept("op", close):
                        break
                    if self.accept("op", ";"):
                        rows.append([])
                        continue
                    if self.accept("op", ","):
                        continue
                    rows[-1].append(self.parse_expr())
                self.index_depth = saved
                rows = [r for r in rows if r]
                return ("matrix" if close == "]" else "cell", rows)
            if t.val == "@":
                name = self.expect("id").val
                return ("fhandle", name)
        raise SyntaxError(f"unexpected token {t!r}")


# ----------------------------------------------------------------------------
# array helpers
# ----------------------------------------------------------------------------

def _broadcast_pair(a, b):
    if a.ndim != b.ndim:
        nd = max(a.ndim, b.ndim)
        a = a.reshape(a.shape + (1,) * (nd - a.ndim))
        b = b.reshape(b.shape + (1,) * (nd - b.ndim))
    return a, b


def _elementwise(f, a, b):
    a, b = _broadcast_pair(_as_float(a), _as_float(b))
    with np.errstate(all="ignore"):
        r = f(a, b)
    return _squeeze_trailing(np.asarray(r))


def _mpower(a, b):
    a = _as_float(a)
    b = _as_float(b)
    a, b = _broadcast_pair(a, b)
    need_c = (not np.iscomplexobj(a) and not np.iscomplexobj(b)
              and np.any((a < 0) & (b != np.round(b))))
    if need_c:
        a = a.astype(complex)
    with np.errstate(all="ignore"):
        r = np.power(a, b)
    return _squeeze_trailing(_realify(np.asarray(r)))


def colon_range(a, s, b):
    """a:s:b with MATLAB's element count (a small tolerance on (b-a)/s)."""
    a, s, b = float(a), float(s), float(b)
    if s == 0 or (s > 0 and a > b) or (s < 0 and a < b):
        return np.zeros((1, 0))
    q = (b - a) / s
    n = int(math.floor(q + 1e-10 * max(1.0, abs(q)))) + 1
    return (a + np.arange(n, dtype=float) * s).reshape(1, n)


def _index_list(ix, extent):
    """One subscript -> 0-based int array."""
    if isinstance(ix, str) and ix == ":":
        return np.arange(extent)
    a = num(ix)
    if a.dtype == bool:
        return np.nonzero(a.reshape(-1, order="F"))[0]
    a = _realify(a)
    if np.iscomplexobj(a):
        raise MatlabError("Subscript indices must either be real positive integers or logicals.")
    flat = a.reshape(-1, order="F")
    r = np.rint(flat)
    if flat.size and (np.any(np.abs(r - flat) > 0) or np.any(r < 1)):
        raise MatlabError("Subscript indices must either be real positive integers or logicals.")
    return r.astype(np.int64) - 1


def do_index(A, subs):
    if isinstance(A, MStr):
        arr = np.array([list(A)], dtype=object) if len(A) else np.zeros((1, 0), dtype=object)
        res = do_index_arr(arr, subs)
        return MStr("".join(res.reshape(-1, order="F")))
    return do_index_arr(num(A), subs)


def do_index_arr(A, subs):
    if len(subs) == 1:
        ix = subs[0]
        flat = A.reshape(-1, order="F")
        idx = _index_list(ix, flat.size)
        if idx.size and idx.max() >= flat.size:
            raise MatlabError("Index exceeds array bounds.")
        vals = flat[idx]
        if isinstance(ix, str):
            return vals.reshape(-1, 1)
        ia = num(ix)
        if ia.dtype == bool:
            # logical mask: column unless A is a row vector
            if A.ndim == 2 and A.shape[0] == 1:
                return vals.reshape(1, -1)
            return vals.reshape(-1, 1)
        is_vec_a = A.ndim == 2 and (A.shape[0] == 1 or A.shape[1] == 1)
        is_vec_i = ia.ndim == 2 and (ia.shape[0] == 1 or ia.shape[1] == 1)
        if is_vec_a and is_vec_i:
            return vals.reshape(1, -1) if A.shape[0] == 1 else vals.reshape(-1, 1)
        return vals.reshape(ia.shape, order="F")
    nd = len(subs)
    shape = list(A.shape)
    if nd < len(shape):
        shape = shape[:nd - 1] + [int(np.prod(shape[nd - 1:]))]
        A = A.reshape(shape, order="F")
    elif nd > len(shape):
        shape = shape + [1] * (nd - len(shape))
        A = A.reshape(shape, order="F")
    idx = [_index_list(s, shape[k]) for k, s in enumerate(subs)]
    for k, ii in enumerate(idx):
        if ii.size and ii.max() >= shape[k]:
            raise MatlabError("Index exceeds matrix dimensions.")
    res = A[np.ix_(*idx)]
    return _squeeze_trailing(res)


def do_assign(A, subs, B):
    """A(subs) = B with growth; returns the new array."""
    if A is None:
        A = np.zeros((0, 0))
    if isinstance(A, MStr):
        A = num(A)
    A = num(A)
    Bv = num(B)
    if np.iscomplexobj(Bv) and not np.iscomplexobj(A):
        A = A.astype(complex)
    elif A.dtype == bool and Bv.dtype != bool:
        A = A.astype(float)
    elif A.dtype != bool and Bv.dtype == bool:
        Bv = Bv.astype(A.dtype)
    if len(subs) == 1:
        ix = subs[0]
        n = A.size
        idx = _index_list(ix, n)
        if idx.size and idx.max() >= n:
            need = int(idx.max()) + 1
            if A.size == 0:
                A = np.zeros((1, need), dtype=A.dtype) if True else A
            elif A.ndim == 2 and A.shape[0] == 1:
                A = np.concatenate([A, np.zeros((1, need - n), dtype=A.dtype)], axis=1)
            elif A.ndim == 2 and A.shape[1] == 1:
                A = np.concatenate([A, np.zeros((need - n, 1), dtype=A.dtype)], axis=0)
            else:
                raise MatlabError("linear index growth of a matrix is not supported")
        flat = A.reshape(-1, order="F").copy()
        bflat = Bv.reshape(-1, order="F")
        if bflat.size == 1:
            flat[idx] = bflat[0]
        elif bflat.size == idx.size:
            flat[idx] = bflat
        else:
            raise MatlabError("In an assignment  A(I) = B, the number of elements in B and I must be the same.")
        return flat.reshape(A.shape, order="F")
    nd = len(subs)
    shape = list(A.shape)
    if nd < len(shape):
        shape = shape[:nd - 1] + [int(np.prod(shape[nd - 1:]))]
        A = A.reshape(shape, order="F")
    elif nd > len(shape):
        shape = shape + [1] * (nd - len(shape))
        A = A.reshape(shape, order="F")
    idx = []
    new_shape = list(shape)
    for k, s in enumerate(subs):
        if isinstance(s, str) and s == ":":
            ext = shape[k]
            if ext == 0:
                # A(:, j) = B on an empty array: the colon takes the elements of B
                # that the other subscripts do not account for
                others = 1
                for kk, ss in enumerate(subs):
                    if kk != k and not (isinstance(ss, str) and ss == ":"):
                        others *= _index_list(ss, shape[kk]).size
                ext = max(Bv.size // max(others, 1), 1)
                new_shape[k] = ext
            idx.append(np.arange(ext))
        else:
            ii = _index_list(s, shape[k])
            idx.append(ii)
            if ii.size and ii.max() + 1 > new_shape[k]:
                new_shape[k] = int(ii.max()) + 1
    if new_shape != shape:
        G = np.zeros(new_shape, dtype=A.dtype)
        G[tuple(slice(0, e) for e in shape)] = A
        A = G
    else:
        A = A.copy()
    target_shape = tuple(len(ii) for ii in idx)
    if Bv.size == 1:
        A[np.ix_(*idx)] = Bv.reshape(-1)[0]
    else:
        if Bv.size != int(np.prod(target_shape)):
            raise MatlabError("Subscripted assignment dimension mismatch.")
        bsq = [d for d in Bv.shape if d != 1]
        tsq = [d for d in target_shape if d != 1]
        if bsq != tsq:
            raise MatlabError("Subscripted assignment dimension mismatch.")
        A[np.ix_(*idx)] = Bv.reshape(-1, order="F").reshape(target_shape, order="F")
    return _squeeze_trailing(A)


# ----------------------------------------------------------------------------
# interpreter
# ----------------------------------------------------------------------------

class Frame:
    def __init__(self, name, nargin, nargout):
        self.vars = {}
        self.name = name
        self.nargin = nargin
        self.nargout = nargout


class Interp:
    def __init__(self, search_path, utape=None, ntape=None):
        self.path = list(search_path)
        self.cache = {}
        self.utape = np.asarray(utape if utape is not None else [], dtype=float).reshape(-1)
        self.ntape = np.asarray(ntape if ntape is not None else [], dtype=float).reshape(-1)
        self.ui = 0
        self.ni = 0
        self.frames = []
        self.end_ctx = []

    # -- files ------------------------------------------------------------
    def find_file(self, name):
        for d in self.path:
            p = os.path.join(d, name + ".m")
            if os.path.exists(p):
                return p
        return None

    def load(self, name):
        if name in self.cache:
            return self.cache[name]
        p = self.find_file(name)
        if p is None:
            return None
        with open(p, encoding="latin-1") as f:
            src = f.read()
        funcs, order = Parser(lex(src)).parse_file()
        # MATLAB dispatches by file name: the first function is the entry
        main = funcs[order[0]]
        self.cache[name] = (main, funcs)
        return self.cache[name]

    # -- random tapes -----------------------------------------------------
    def draw(self, which, shape):
        n = int(np.prod(shape)) if shape else 1
        if which == "u":
            if self.ui + n > self.utape.size:
                raise MatlabError("rand tape exhausted")
            v = self.utape[self.ui:self.ui + n]
            self.ui += n
        else:
            if self.ni + n > self.ntape.size:
                raise MatlabError("randn tape exhausted")
            v = self.ntape[self.ni:self.ni + n]
            self.ni += n
        return M(v.reshape(shape, order="F"))

    # -- calls ------------------------------------------------------------
    def call(self, name, args, nargout=1):
        ent = self.load(name)
        if ent is not None:
            main, funcs = ent
            return self.run_function(main, funcs, args, nargout)
        if name in BUILTINS:
            res = BUILTINS[name](self, args, nargout)
            if not isinstance(res, list):
                res = [res]
            return res
        raise MatlabError(f"Undefined function or variable '{name}'.")

    def run_function(self, f, local_funcs, args, nargout):
        if len(args) > len(f["params"]) and not (f["params"] and f["params"][-1] == "varargin"):
            raise MatlabError("Too many input arguments.")
        fr = Frame(f["name"], len(args), nargout)
        fr.local_funcs = local_funcs
        ps = f["params"]
        for k, a in enumerate(args):
            if ps[k] == "varargin" and k == len(ps) - 1:
                fr.vars["varargin"] = MCell(args[k:])
                break
            if ps[k] != "~":
                fr.vars[ps[k]] = a
        if ps and ps[-1] == "varargin" and "varargin" not in fr.vars:
            fr.vars["varargin"] = MCell([])
        self.frames.append(fr)
        try:
            self.exec_block(f["body"])
        except _Return:
            pass
        finally:
            self.frames.pop()
        outs = []
        for k, o in enumerate(f["outs"][:max(nargout, 1)]):
            if o not in fr.vars:
                if k < nargout:
                    raise MatlabError(f"Output argument \"{o}\" (and maybe others) not assigned during call to \"{f['name']}\".")
                break
            outs.append(fr.vars[o])
        return outs

    @property
    def fr(self):
        return self.frames[-1]

    # -- statements -------------------------------------------------------
    def exec_block(self, stmts):
        for s in stmts:
            self.exec_stmt(s)

    def exec_stmt(self, s):
        k = s[0]
        if k == "expr":
            e = s[1]
            if e[0] == "id" and e[1] not in self.fr.vars:
                self.call_named(e[1], [], 0)
            elif e[0] == "call" and e[1][0] == "id" and e[1][1] not in self.fr.vars:
                args = [self.eval_arg(a) for a in e[2]]
                self.call_named(e[1][1], args, 0)
            else:
                self.eval(e)
        elif k == "assign":
            self.assign(s[1], self.eval(s[2]))
        elif k == "massign":
            targets, rhs = s[1], s[2]
            if rhs[0] == "call" and rhs[1][0] == "id" and rhs[1][1] not in self.fr.vars:
                args = [self.eval_arg(a) for a in rhs[2]]
                vals = self.call_named(rhs[1][1], args, len(targets))
            elif rhs[0] == "id" and rhs[1] not in self.fr.vars:
                vals = self.call_named(rhs[1], [], len(targets))
            else:
                vals = [self.eval(rhs)]
            for t, v in zip(targets, vals):
                if t is not None:
                    self.assign(t, v)
        elif k == "if":
            for cond, body in s[1]:
                if self.cond(cond):
                    self.exec_block(body)
                    return
            if s[2] is not None:
                self.exec_block(s[2])
        elif k == "for":
            rng = self.eval(s[2])
            arr = num(rng)
            ncols = arr.shape[1] if arr.ndim >= 2 else arr.size
            if arr.ndim > 2:
                arr = arr.reshape(arr.shape[0], -1, order="F")
                ncols = arr.shape[1]
            for c in range(ncols):
                self.fr.vars[s[1]] = M(arr[:, c:c + 1])
                try:
                    self.exec_block(s[3])
                except _Break:
                    break
                except _Continue:
                    continue
        elif k == "while":
            while self.cond(s[1]):
                try:
                    self.exec_block(s[2])
                except _Break:
                    break
                except _Continue:
                    continue
        elif k == "switch":
            subj = self.eval(s[1])
            for val, body in s[2]:
                v = self.eval(val)
                if self.switch_match(subj, v):
                    self.exec_block(body)
                    return
            if s[3] is not None:
                self.exec_block(s[3])
        elif k == "break":
            raise _Break()
        elif k == "continue":
            raise _Continue()
        elif k == "return":
            raise _Return()
        else:
            raise RuntimeError(f"unknown statement {k}")

    def switch_match(self, subj, v):
        if isinstance(v, MCell):
            return any(self.switch_match(subj, x) for x in v.items)
        if isinstance(subj, MStr) or isinstance(v, MStr):
            return isinstance(subj, MStr) and isinstance(v, MStr) and str(subj) == str(v)
        return scalar(subj) == scalar(v)

    def cond(self, e):
        """if / while condition: & and | short-circuit here."""
        if e[0] == "bin" and e[1] in ("&", "|", "&&", "||"):
            left = self.cond(e[2])
            if e[1] in ("&", "&&") and not left:
                return False
            if e[1] in ("|", "||") and left:
                return True
            return self.cond(e[3])
        if e[0] == "paren":
            return self.cond(e[1])
        return truth(self.eval(e))

    def call_named(self, name, args, nargout):
        fr = self.frames[-1] if self.frames else None
        if fr is not None and getattr(fr, "local_funcs", None) and name in fr.local_funcs and self.load(name) is None:
            return self.run_function(fr.local_funcs[name], fr.local_funcs, args, nargout)
        return self.call(name, args, nargout)

    # -- assignment -------------------------------------------------------
    def assign(self, target, value):
        if isinstance(value, np.ndarray):
            value = _squeeze_trailing(value)
        if target[0] == "id":
            self.fr.vars[target[1]] = value
            return
        base, chain = self.flatten_lvalue(target)
        cur = self.fr.vars.get(base)
        self.fr.vars[base] = self.assign_chain(cur, chain, value)

    def flatten_lvalue(self, e):
        chain = []
        while e[0] != "id":
            if e[0] == "call":
                chain.append(("()", e[2]))
                e = e[1]
            elif e[0] == "field":
                chain.append((".", e[2]))
                e = e[1]
            elif e[0] == "cellidx":
                chain.append(("{}", e[2]))
                e = e[1]
            else:
                raise SyntaxError("bad assignment target")
        return e[1], list(reversed(chain))

    def assign_chain(self, cur, chain, value):
        kind, arg = chain[0]
        rest = chain[1:]
        if kind == ".":
            st = cur if isinstance(cur, MStruct) else MStruct()
            st = MStruct(st)
            if rest:
                st[arg] = self.assign_chain(st.get(arg), rest, value)
            else:
                st[arg] = value
            return st
        if kind == "{}":
            cell = cur if isinstance(cur, MCell) else MCell([])
            subs = [self.eval_index(a, cell.items, k, len(arg)) for k, a in enumerate(arg)]
            idx = int(scalar(subs[-1])) - 1
            items = list(cell.items)
            while len(items) <= idx:
                items.append(M(np.zeros((0, 0))))
            items[idx] = value if not rest else self.assign_chain(items[idx], rest, value)
            return MCell(items)
        # "()"
        if rest:
            raise MatlabError("nested indexed assignment not supported")
        arr = cur if cur is not None else np.zeros((0, 0))
        subs = [self.eval_index(a, arr, k, len(arg)) for k, a in enumerate(arg)]
        return do_assign(arr, subs, value)

    # -- expressions ------------------------------------------------------
    def eval_arg(self, e):
        return self.eval(e)

    def eval_index(self, e, arr, k, n):
        if e[0] == "colon_all":
            return ":"
        self.end_ctx.append((arr, k, n))
        try:
            return self.eval(e)
        finally:
            self.end_ctx.pop()

    def end_value(self):
        arr, k, n = self.end_ctx[-1]
        if isinstance(arr, list):
            return M(float(len(arr)))
        if isinstance(arr, MStr):
            sz = [1, len(arr)]
        else:
            sz = list(num(arr).shape)
        if n == 1:
            return M(float(np.prod(sz)))
        if k < n - 1:
            return M(float(sz[k] if k < len(sz) else 1))
        return M(float(np.prod(sz[k:])) if k < len(sz) else 1.0)

    def eval(self, e):
        k = e[0]
        if k == "num":
            return M(e[1])
        if k == "str":
            return MStr(e[1])
        if k == "paren":
            return self.eval(e[1])
        if k == "end":
            return self.end_value()
        if k == "id":
            name = e[1]
            if name in self.fr.vars:
                return self.fr.vars[name]
            r = self.call_named(name, [], 1)
            if not r:
                raise MatlabError(f"{name} returned no value")
            return r[0]
        if k == "call":
            base = e[1]
            if base[0] == "id" and base[1] not in self.fr.vars:
                args = [self.eval_arg(a) for a in e[2]]
                r = self.call_named(base[1], args, 1)
                if not r:
                    raise MatlabError(f"{base[1]} returned no value")
                return r[0]
            arr = self.eval(base)
            if isinstance(arr, FHandle):
                args = [self.eval_arg(a) for a in e[2]]
                return self.call(arr.name, args, 1)[0]
            subs = [self.eval_index(a, arr, j, len(e[2])) for j, a in enumerate(e[2])]
            return do_index(arr, subs)
        if k == "cellidx":
            cell = self.eval(e[1])
            subs = [self.eval_index(a, cell.items, j, len(e[2])) for j, a in enumerate(e[2])]
            return cell.items[int(scalar(subs[-1])) - 1]
        if k == "field":
            st = self.eval(e[1])
            if not isinstance(st, MStruct):
                raise MatlabError("Attempt to reference field of non-structure array.")
            if e[2] not in st:
                raise MatlabError(f"Reference to non-existent field '{e[2]}'.")
            return st[e[2]]
        if k == "ctranspose":
            a = self.eval(e[1])
            if isinstance(a, MStr):
                return a
            return _squeeze_trailing(np.conj(num(a)).T.copy())
        if k == "transpose":
            return num(self.eval(e[1])).T.copy()
        if k == "un":
            a = self.eval(e[2])
            if e[1] == "-":
                return M(-_as_float(a))
            if e[1] == "+":
                return a
            return M(~(num(a) != 0))
        if k == "bin":
            return self.binop(e[1], e[2], e[3])
        if k == "range":
            a = scalar(self.eval(e[1]))
            s = 1.0 if e[2] is None else scalar(self.eval(e[2]))
            b = scalar(self.eval(e[3]))
            return colon_range(np.real(a), np.real(s), np.real(b))
        if k == "matrix":
            return self.build_matrix(e[1])
        if k == "cell":
            return MCell([self.eval(x) for row in e[1] for x in row])
        if k == "fhandle":
            return FHandle(e[1])
        if k == "colon_all":
            return MStr(":")
        raise RuntimeError(f"unknown expression {k}")

    def build_matrix(self, rows):
        built = []
        for row in rows:
            vals = [self.eval(x) for x in row]
            if vals and all(isinstance(v, MStr) for v in vals):
                built.append(MStr("".join(vals)))
                continue
            arrs = [num(v) for v in vals]
            arrs = [a for a in arrs if a.size > 0 or a.shape[0] > 0]
            arrs = [a for a in arrs if a.size > 0]
            if not arrs:
                built.append(np.zeros((0, 0)))
                continue
            built.append(np.concatenate(arrs, axis=1) if len(arrs) > 1 else arrs[0])
        if len(built) == 1 and isinstance(built[0], MStr):
            return built[0]
        built = [num(b) for b in built if num(b).size > 0]
        if not built:
            return np.zeros((0, 0))
        if any(np.iscomplexobj(b) for b in built):
            built = [b.astype(complex) for b in built]
        elif any(b.dtype != bool for b in built):
            built = [b.astype(float) if b.dtype == bool else b for b in built]
        return _squeeze_trailing(np.concatenate(built, axis=0) if len(built) > 1 else built[0])

    def binop(self, op, le, re_):
        if op == "&&":
            return M(truth(self.eval(le)) and truth(self.eval(re_)))
        if op == "||":
            return M(truth(self.eval(le)) or truth(self.eval(re_)))
        return self.binop_values(op, self.eval(le), self.eval(re_))

    def binop_values(self, op, a, b):
        if op in ("==", "~=") and (isinstance(a, MStr) or isinstance(b, MStr)):
            a, b = num(a), num(b)
        an, bn = num(a), num(b)
        if op == "+":
            return _realify(_elementwise(np.add, an, bn))
        if op == "-":
            return _realify(_elementwise(np.subtract, an, bn))
        if op == ".*":
            return _realify(_elementwise(np.multiply, an, bn))
        if op == "./":
            return _realify(_elementwise(np.divide, an, bn))
        if op == ".\\":
            return _realify(_elementwise(np.divide, bn, an))
        if op == "*":
            if an.size == 1 or bn.size == 1:
                return _realify(_elementwise(np.multiply, an, bn))
            A, B = _as_float(an), _as_float(bn)
            if A.ndim != 2 or B.ndim != 2 or A.shape[1] != B.shape[0]:
                raise MatlabError("Inner matrix dimensions must agree.")
            return _realify(A @ B)
        if op == "/":
            if bn.size == 1:
                return _realify(_elementwise(np.divide, an, bn))
            A, B = _as_float(an), _as_float(bn)
            return _realify(np.linalg.lstsq(B.T, A.T, rcond=None)[0].T)
        if op == "\\":
            if an.size == 1:
                return _realify(_elementwise(np.divide, bn, an))
            A, B = _as_float(an), _as_float(bn)
            return _realify(np.linalg.solve(A, B))
        if op == ".^":
            return _mpower(an, bn)
        if op == "^":
            if an.size == 1 and bn.size == 1:
                return _mpower(an, bn)
            raise MatlabError("matrix power not supported")
        if op in ("==", "~=", "<", "<=", ">", ">="):
            f = {"==": np.equal, "~=": np.not_equal, "<": np.less, "<=": np.less_equal,
                 ">": np.greater, ">=": np.greater_equal}[op]
            A, B = _as_float(an), _as_float(bn)
            if op not in ("==", "~="):
                A = A.real if np.iscomplexobj(A) else A
                B = B.real if np.iscomplexobj(B) else B
            return _elementwise(f, A, B)
        if op == "&":
            return _elementwise(np.logical_and, an != 0, bn != 0)
        if op == "|":
            return _elementwise(np.logical_or, an != 0, bn != 0)
        raise RuntimeError(f"unknown operator {op}")


# ----------------------------------------------------------------------------
# builtins
# ----------------------------------------------------------------------------

def _dims_from_args(args):
    if not args:
        return (1, 1)
    if len(args) == 1:
        a = num(args[0]).reshape(-1)
        if a.size == 1:
            n = int(a[0])
            return (n, n)
        return tuple(int(x) for x in a)
    return tuple(int(scalar(x)) for x in args)


def _fill(val):
    def f(it, args, nargout):
        args = [a for a in args if not isinstance(a, MStr)]
        shp = _dims_from_args(args)
        shp = tuple(max(d, 0) for d in shp)
        return _squeeze_trailing(np.full(shp, val, dtype=float))
    return f


def _first_nonsingleton(a):
    for k, d in enumerate(a.shape):
        if d != 1:
            return k
    return 0


def _reduce(fn):
    def f(it, args, nargout):
        a = _as_float(args[0])
        if len(args) > 1:
            dim = int(scalar(args[1])) - 1
        else:
            dim = _first_nonsingleton(a)
        if a.size == 0 and len(args) == 1 and a.shape == (0, 0):
            return M(fn(np.zeros(0)))
        if dim >= a.ndim:
            return a
        return _squeeze_trailing(_realify(np.expand_dims(fn(a, axis=dim), dim)))
    return f


def _minmax(which):
    pick = np.argmin if which == "min" else np.argmax

    def f(it, args, nargout):
        if len(args) >= 2 and num(args[1]).size > 0:
            a, b = _as_float(args[0]), _as_float(args[1])
            fn = np.fmin if which == "min" else np.fmax
            return _elementwise(fn, a, b)
        a = _as_float(args[0])
        dim = int(scalar(args[2])) - 1 if len(args) >= 3 else _first_nonsingleton(a)
        key = np.abs(a) if np.iscomplexobj(a) else a
        key = np.where(np.isnan(key), np.inf if which == "min" else -np.inf, key)
        idx = pick(key, axis=dim)
        vals = np.take_along_axis(a, np.expand_dims(idx, dim), axis=dim)
        out = [_squeeze_trailing(vals)]
        if nargout > 1:
            out.append(_squeeze_trailing(np.expand_dims(idx, dim).astype(float) + 1))
        return out
    return f


def _mround(x):
    x = _as_float(x)
    if np.iscomplexobj(x):
        return _realify(_mround(x.real) + 1j * _mround(x.imag))
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def _auto_complex(fn, bad):
    def f(it, args, nargout):
        a = _as_float(args[0])
        if not np.iscomplexobj(a) and np.any(bad(a)):
            a = a.astype(complex)
        with np.errstate(all="ignore"):
            return _squeeze_trailing(_realify(fn(a)))
    return f


def _elem(fn):
    def f(it, args, nargout):
        with np.errstate(all="ignore"):
            return _squeeze_trailing(_realify(np.asarray(fn(_as_float(args[0])))))
    return f


def b_size(it, args, nargout):
    a = args[0]
    shp = [1, len(a)] if isinstance(a, MStr) else ([1, len(a.items)] if isinstance(a, MCell) else
                                                   ([1, 1] if isinstance(a, (MStruct, FHandle)) else list(num(a).shape)))
    if len(args) > 1:
        d = int(scalar(args[1]))
        return M(float(shp[d - 1] if d - 1 < len(shp) else 1))
    if nargout <= 1:
        return M(np.array(shp, dtype=float))
    out = [M(float(s)) for s in shp[:nargout - 1]]
    out.append(M(float(np.prod(shp[nargout - 1:]))))
    while len(out) < nargout:
        out.append(M(1.0))
    return out


def _numel(a):
    if isinstance(a, MStr):
        return len(a)
    if isinstance(a, MCell):
        return len(a.items)
    if isinstance(a, (MStruct, FHandle)):
        return 1
    return num(a).size


def b_length(it, args, nargout):
    a = args[0]
    if isinstance(a, MStr):
        return M(float(len(a)))
    if isinstance(a, MCell):
        return M(float(len(a.items)))
    s = num(a).shape
    return M(float(0 if num(a).size == 0 else max(s)))


def b_rand(which):
    def f(it, args, nargout):
        args = [a for a in args if not isinstance(a, MStr)]
        shp = _dims_from_args(args)
        return it.draw(which, shp)
    return f


def b_exist(it, args, nargout):
    name = str(args[0])
    kind = str(args[1]) if len(args) > 1 else ""
    if name in it.fr.vars:
        return M(1.0)
    if kind == "var":
        return M(0.0)
    if it.find_file(name):
        return M(2.0)
    return M(5.0 if name in BUILTINS else 0.0)


def b_error(it, args, nargout):
    msg = str(args[0]) if args else ""
    if len(args) > 1 and ":" in msg and " " not in msg:
        msg = str(args[1])
    raise MatlabError(msg)


def b_narginchk(it, args, nargout):
    lo, hi = scalar(args[0]), scalar(args[1])
    n = it.fr.nargin
    if n < lo:
        raise MatlabError("Not enough input arguments.")
    if n > hi:
        raise MatlabError("Too many input arguments.")
    return []


def b_norm(it, args, nargout):
    a = _as_float(args[0])
    if a.ndim == 2 and min(a.shape) == 1 or a.size <= 1:
        return M(float(np.sqrt(np.sum(np.abs(a) ** 2))))
    return M(float(np.linalg.norm(a, 2)))


def b_repmat(it, args, nargout):
    a = num(args[0])
    reps = _dims_from_args(args[1:])
    a2 = a.reshape(a.shape + (1,) * (len(reps) - a.ndim)) if len(reps) > a.ndim else a
    reps2 = tuple(reps) + (1,) * (a2.ndim - len(reps))
    return _squeeze_trailing(np.tile(a2, reps2))


def b_reshape(it, args, nargout):
    a = num(args[0])
    dims = list(_dims_from_args(args[1:])) if len(args) > 2 else [int(x) for x in num(args[1]).reshape(-1)]
    return _squeeze_trailing(a.reshape(dims, order="F"))


def b_find(it, args, nargout):
    a = num(args[0])
    idx = np.nonzero(a.reshape(-1, order="F"))[0] + 1.0
    if len(args) > 1:
        idx = idx[: int(scalar(args[1]))]
    if a.ndim == 2 and a.shape[0] == 1:
        return M(idx.reshape(1, -1))
    return idx.reshape(-1, 1)


def b_cumsum(it, args, nargout):
    a = _as_float(args[0])
    dim = int(scalar(args[1])) - 1 if len(args) > 1 else _first_nonsingleton(a)
    return np.cumsum(a, axis=dim)


def b_diff(it, args, nargout):
    a = _as_float(args[0])
    dim = int(scalar(args[2])) - 1 if len(args) > 2 else _first_nonsingleton(a)
    return np.diff(a, axis=dim)


def b_allany(fn):
    def f(it, args, nargout):
        a = num(args[0]) != 0
        dim = int(scalar(args[1])) - 1 if len(args) > 1 else _first_nonsingleton(a)
        if a.size == 0:
            return M(fn(np.zeros(0, dtype=bool)))
        return _squeeze_trailing(np.expand_dims(fn(a, axis=dim), dim))
    return f


def b_mean(it, args, nargout):
    a = _as_float(args[0])
    dim = int(scalar(args[1])) - 1 if len(args) > 1 else _first_nonsingleton(a)
    return _squeeze_trailing(_realify(np.expand_dims(np.sum(a, axis=dim) / a.shape[dim], dim)))


def b_median(it, args, nargout):
    a = _as_float(args[0])
    dim = _first_nonsingleton(a)
    return _squeeze_trailing(np.expand_dims(np.median(a, axis=dim), dim))


def b_sort(it, args, nargout):
    a = _as_float(args[0])
    dim = _first_nonsingleton(a)
    idx = np.argsort(a, axis=dim, kind="stable")
    vals = np.take_along_axis(a, idx, axis=dim)
    return [vals, idx.astype(float) + 1][:max(nargout, 1)]


def b_linspace(it, args, nargout):
    a, b = scalar(args[0]), scalar(args[1])
    n = int(scalar(args[2])) if len(args) > 2 else 100
    return M(np.linspace(a, b, n).reshape(1, n))


def b_ndgrid(it, args, nargout):
    vs = [num(a).reshape(-1, order="F") for a in args]
    if len(vs) == 1:
        vs = vs * max(nargout, 2)
    grids = np.meshgrid(*vs, indexing="ij")
    return [_squeeze_trailing(g) for g in grids][:max(nargout, 1)]


def b_meshgrid(it, args, nargout):
    vs = [num(a).reshape(-1, order="F") for a in args]
    if len(vs) == 1:
        vs = vs * 2
    grids = np.meshgrid(*vs, indexing="xy")
    return [_squeeze_trailing(g) for g in grids][:max(nargout, 1)]


def b_padarray(it, args, nargout):
    a = num(args[0])
    pad = [int(x) for x in num(args[1]).reshape(-1)]
    if any(float(x) != int(x) for x in num(args[1]).reshape(-1)):
        raise MatlabError("PADSIZE must be a vector of nonnegative integers.")
    mode = str(args[2]) if len(args) > 2 else "both"
    width = []
    for k in range(a.ndim):
        p = pad[k] if k < len(pad) else 0
        width.append((p, p) if mode == "both" else ((p, 0) if mode == "pre" else (0, p)))
    return np.pad(a, width)


def b_fft2(it, args, nargout):
    return _realify(np.fft.fft2(_as_float(args[0]), axes=(0, 1)))


def b_strcmp(it, args, nargout):
    a, b = args[0], args[1]
    return M(isinstance(a, MStr) and isinstance(b, MStr) and str(a) == str(b))


def b_strncmpi(it, args, nargout):
    a, b, n = str(args[0]), str(args[1]), int(scalar(args[2]))
    return M(len(a) >= n and len(b) >= n and a[:n].lower() == b[:n].lower())


def b_isfield(it, args, nargout):
    return M(isinstance(args[0], MStruct) and str(args[1]) in args[0])


def b_isscalar(it, args, nargout):
    return M(_numel(args[0]) == 1)


def b_isvector(it, args, nargout):
    a = args[0]
    if isinstance(a, MStr):
        return M(len(a) >= 1)
    s = num(a).shape
    return M(len(s) == 2 and min(s) == 1 and num(a).size >= 1)


def b_isempty(it, args, nargout):
    return M(_numel(args[0]) == 0)


def b_islogical(it, args, nargout):
    a = args[0]
    return M(isinstance(a, np.ndarray) and a.dtype == bool)


def b_isreal(it, args, nargout):
    a = args[0]
    return M(not (isinstance(a, np.ndarray) and np.iscomplexobj(a)))


def b_isnumeric(it, args, nargout):
    a = args[0]
    return M(isinstance(a, np.ndarray) and a.dtype != bool)


def b_hist(it, args, nargout):
    """hist(y, N): counts in N equal-width bins between min(y) and max(y)
    ([e_k, e_k+1), last bin closed) - MATLAB's documented binning."""
    y = _as_float(args[0]).reshape(-1, order="F")
    n = int(scalar(args[1])) if len(args) > 1 else 10
    lo, hi = float(np.min(y)), float(np.max(y))
    if hi == lo:
        counts = np.zeros(n)
        counts[0] = y.size
    else:
        counts, _ = np.histogram(y, bins=n, range=(lo, hi))
    return M(counts.astype(float).reshape(1, -1))


def b_sinc(it, args, nargout):
    return np.sinc(_as_float(args[0]))


def b_null(it, args, nargout):
    a = _as_float(args[0])
    u, s, vh = np.linalg.svd(a)
    tol = max(a.shape) * (s[0] if s.size else 0) * np.finfo(float).eps
    r = int(np.sum(s > tol))
    return vh[r:].conj().T


def b_mod(it, args, nargout):
    a, b = _as_float(args[0]), _as_float(args[1])
    return _elementwise(lambda x, y: np.where(y == 0, x, x - np.floor(x / np.where(y == 0, 1, y)) * y), a, b)


def b_rem(it, args, nargout):
    a, b = _as_float(args[0]), _as_float(args[1])
    return _elementwise(lambda x, y: np.where(y == 0, x, x - np.trunc(x / np.where(y == 0, 1, y)) * y), a, b)


def b_num2str(it, args, nargout):
    """num2str of a real scalar (only used here to build progress messages)."""
    v = num(args[0]).reshape(-1)
    if v.size == 1:
        x = float(np.real(v[0]))
        return MStr(str(int(x)) if x == int(x) else f"{x:.4g}")
    return MStr(" ".join(f"{float(np.real(x)):.4g}" for x in v))


def b_char(it, args, nargout):
    a = args[0]
    if isinstance(a, MStr):
        return a
    return MStr("".join(chr(int(x)) for x in num(a).reshape(-1)))


def b_bsxfun(it, args, nargout):
    h = args[0]
    return it.call(h.name, [args[1], args[2]], 1)[0]


def _binop_builtin(op):
    def f(it, args, nargout):
        return it.binop_values(op, args[0], args[1])
    return f


def b_nargin(it, args, nargout):
    return M(float(it.fr.nargin))


def b_nargout(it, args, nargout):
    return M(float(it.fr.nargout))


def b_noop(it, args, nargout):
    return []


def b_abs(it, args, nargout):
    return np.abs(_as_float(args[0]))


def b_angle(it, args, nargout):
    return np.angle(_as_float(args[0]))


def b_real(it, args, nargout):
    return np.real(_as_float(args[0])).copy()


def b_imag(it, args, nargout):
    return np.imag(_as_float(args[0])).copy()


def b_conj(it, args, nargout):
    return np.conj(_as_float(args[0]))


def b_fliplr(it, args, nargout):
    return num(args[0])[:, ::-1].copy()


def b_flipud(it, args, nargout):
    return num(args[0])[::-1].copy()


def b_fftshift(it, args, nargout):
    return np.fft.fftshift(num(args[0]), axes=(0, 1))


def b_ifftshift(it, args, nargout):
    return np.fft.ifftshift(num(args[0]), axes=(0, 1))


def b_prod(it, args, nargout):
    return _reduce(np.prod)(it, args, nargout)


def b_logical(it, args, nargout):
    return num(args[0]) != 0


def b_double(it, args, nargout):
    return _as_float(args[0]).astype(complex if np.iscomplexobj(num(args[0])) else float)


def _const(v):
    def f(it, args, nargout):
        return M(v)
    return f


def b_sign(it, args, nargout):
    return np.sign(_as_float(args[0]))


def b_isinf(it, args, nargout):
    return np.isinf(_as_float(args[0]))


def b_isnan(it, args, nargout):
    return np.isnan(_as_float(args[0]))


def b_max(it, args, nargout):
    return _minmax("max")(it, args, nargout)


def b_min(it, args, nargout):
    return _minmax("min")(it, args, nargout)


BUILTINS = {
    "zeros": _fill(0.0), "ones": _fill(1.0), "inf": _fill(np.inf), "Inf": _fill(np.inf),
    "nan": _fill(np.nan), "NaN": _fill(np.nan),
    "pi": _const(math.pi), "eps": _const(np.finfo(float).eps),
    "i": _const(1j), "j": _const(1j),
    "true": _const(True), "false": _const(False),
    "size": b_size, "numel": lambda it, a, n: M(float(_numel(a[0]))), "length": b_length,
    "ndims": lambda it, a, n: M(float(max(2, num(a[0]).ndim))),
    "isempty": b_isempty, "exist": b_exist, "nargin": b_nargin, "nargout": b_nargout,
    "narginchk": b_narginchk, "error": b_error, "warning": b_noop, "disp": b_noop,
    "fprintf": b_noop, "figure": b_noop, "tic": b_noop, "toc": b_noop, "rng": b_noop,
    "abs": b_abs, "sqrt": _auto_complex(np.sqrt, lambda a: a < 0),
    "exp": _elem(np.exp), "log": _auto_complex(np.log, lambda a: a < 0),
    "sin": _elem(np.sin), "cos": _elem(np.cos), "tan": _elem(np.tan), "atan": _elem(np.arctan),
    "acos": _auto_complex(np.arccos, lambda a: np.abs(a) > 1),
    "asin": _auto_complex(np.arcsin, lambda a: np.abs(a) > 1),
    "atan2": lambda it, a, n: _elementwise(np.arctan2, _as_float(a[0]), _as_float(a[1])),
    "real": b_real, "imag": b_imag, "conj": b_conj, "angle": b_angle,
    "round": lambda it, a, n: _mround(a[0]), "ceil": _elem(np.ceil), "floor": _elem(np.floor),
    "fix": _elem(np.trunc), "mod": b_mod, "rem": b_rem, "sign": b_sign,
    "min": b_min, "max": b_max, "sum": _reduce(np.sum), "prod": b_prod, "mean": b_mean,
    "median": b_median, "cumsum": b_cumsum, "diff": b_diff,
    "all": b_allany(np.all), "any": b_allany(np.any), "find": b_find, "norm": b_norm,
    "repmat": b_repmat, "reshape": b_reshape, "linspace": b_linspace, "ndgrid": b_ndgrid,
    "meshgrid": b_meshgrid, "sort": b_sort, "fliplr": b_fliplr, "flipud": b_flipud,
    "fft2": b_fft2, "fftshift": b_fftshift, "ifftshift": b_ifftshift, "padarray": b_padarray,
    "rand": b_rand("u"), "randn": b_rand("n"), "bsxfun": b_bsxfun,
    "isscalar": b_isscalar, "isvector": b_isvector, "isreal": b_isreal, "isnumeric": b_isnumeric,
    "islogical": b_islogical, "isinf": b_isinf, "isnan": b_isnan, "isfield": b_isfield,
    "hist": b_hist, "strcmp": b_strcmp, "strncmpi": b_strncmpi, "char": b_char, "sinc": b_sinc, "null": b_null,
    "logical": b_logical, "double": b_double, "num2str": b_num2str,
    "deg2rad": lambda it, a, n: _as_float(a[0]) * (math.pi / 180.0),
    "rad2deg": lambda it, a, n: _as_float(a[0]) * (180.0 / math.pi),
    "plus": _binop_builtin("+"), "minus": _binop_builtin("-"), "times": _binop_builtin(".*"),
    "rdivide": _binop_builtin("./"), "power": _binop_builtin(".^"),
    "gt": _binop_builtin(">"), "ge": _binop_builtin(">="), "lt": _binop_builtin("<"),
    "le": _binop_builtin("<="), "eq": _binop_builtin("=="),
}


def reference_search_path(ref_root):
    """The folders scmc.m puts on MATLAB's path (code/, coreFunctions, interface/*)."""
    return [
        ref_root,
        os.path.join(ref_root, "code"),
        os.path.join(ref_root, "code", "coreFunctions"),
        os.path.join(ref_root, "interface", "scatter"),
        os.path.join(ref_root, "interface", "source"),
        os.path.join(ref_root, "interface", "targetArea"),
    ]
