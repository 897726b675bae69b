"""Mechanical evaluator for the Fortran subset of seiya/scale-dg-kernel-extraction.

It translates the reference's own source files (main.f90, mod_common.f90,
mod_mesh.f90, mod_advect3d_eq.f90, mod_dg_optr_kernel.f90 and the generated
mod_dg_optr_kernel_opt1.f90) statement by statement into Python and runs
them, so that golden vectors come from the reference's code text rather
than from a hand restatement.  No Fortran compiler exists in this image;
this is the closest stand-in for running the reference itself.

Fidelity: every real expression is emitted fully parenthesised in Fortran's
precedence and left-to-right order and evaluated in IEEE double precision
(Python floats, or numpy float64 element-wise for array syntax), which is
what an x86-64 gfortran build without FMA computes.  Scalar intrinsics call
the C math library (math.sin etc.), like gfortran.  Supported: modules,
subroutines, functions, the main program, explicit-shape and allocatable
arrays with sections and vector subscripts, sequence association of array
arguments, do / if / select case, list-directed and namelist reads,
formatted writes of the formats the reference uses.  The Timer type is
replaced by a stub (its values never reach the numerics).

Used only by make_golden.py to produce fixtures; nothing at test time reads
the reference.
"""
import math
import os
import re

import numpy as np

# ---------------------------------------------------------------------------
# Runtime
# ---------------------------------------------------------------------------


class FortranStop(Exception):
    pass


class Colon:
    """A section subscript lo:hi (None = the array bound)."""

    __slots__ = ("lo", "hi")

    def __init__(self, lo=None, hi=None):
        self.lo, self.hi = lo, hi


class FArr:
    """Column-major array with 1-based indices over a flat numpy buffer."""

    __slots__ = ("buf", "off", "dims", "strides", "size")

    def __init__(self, buf, off, dims):
        self.buf, self.off, self.dims = buf, off, tuple(int(d) for d in dims)
        st, s = [], 1
        for d in self.dims:
            st.append(s)
            s *= d
        self.strides, self.size = tuple(st), s

    @staticmethod
    def zeros(dims, dtype):
        n = 1
        for d in dims:
            n *= int(d)
        return FArr(np.zeros(n, dtype=dtype), 0, dims)

    def view(self, dims):
        return FArr(self.buf, self.off, dims)

    def flat(self):
        return self.buf[self.off:self.off + self.size]

    def _axes(self, ix):
        axes, scalar = [], True
        for d, i in enumerate(ix):
            if isinstance(i, Colon):
                lo = 1 if i.lo is None else int(i.lo)
                hi = self.dims[d] if i.hi is None else int(i.hi)
                axes.append(np.arange(lo, hi + 1))
                scalar = False
            elif isinstance(i, np.ndarray):
                axes.append(i.astype(np.int64))
                scalar = False
            else:
                axes.append(np.array([int(i)]))
        return axes, scalar

    def _lin(self, axes):
        """Flat buffer positions of a section, first subscript fastest."""
        grids = np.meshgrid(*axes, indexing="ij")
        lin = np.full(grids[0].shape, self.off, dtype=np.int64)
        for g, st in zip(grids, self.strides):
            lin += (g - 1) * st
        return lin.reshape(-1, order="F")

    def get(self, *ix):
        if all(isinstance(i, (int, np.integer)) for i in ix):
            n = self.off
            for d, i in enumerate(ix):
                n += (int(i) - 1) * self.strides[d]
            v = self.buf[n]
            return float(v) if self.buf.dtype.kind == "f" else int(v)
        axes, _ = self._axes(ix)
        return self.buf[self._lin(axes)].copy()

    def set(self, val, *ix):
        if isinstance(val, FArr):
            val = val.flat().copy()
        if not ix:
            self.buf[self.off:self.off + self.size] = val
            return
        if all(isinstance(i, (int, np.integer)) for i in ix):
            n = self.off
            for d, i in enumerate(ix):
                n += (int(i) - 1) * self.strides[d]
            self.buf[n] = val
            return
        axes, _ = self._axes(ix)
        self.buf[self._lin(axes)] = val

    def section_view(self, ix):
        """A view for a contiguous section a(:, j, k) passed as an actual."""
        if not ix:
            return self
        n_colon = 0
        for i in ix:
            if isinstance(i, Colon):
                if i.lo is not None or i.hi is not None:
                    return None
                n_colon += 1
            elif not isinstance(i, (int, np.integer)):
                return None
        # leading full colons followed by scalars is contiguous
        seen_scalar = False
        for i in ix:
            if isinstance(i, Colon):
                if seen_scalar:
                    return None
            else:
                seen_scalar = True
        off = self.off
        for d, i in enumerate(ix):
            if not isinstance(i, Colon):
                off += (int(i) - 1) * self.strides[d]
        return FArr(self.buf, off, self.dims[:n_colon] if n_colon else (1,))


def val(x):
    """Value of an array operand in an expression (whole array -> flat)."""
    return x.flat().copy() if isinstance(x, FArr) else x


class Ref:
    """A scalar passed by reference."""

    __slots__ = ("scope", "name")

    def __init__(self, scope, name):
        self.scope, self.name = scope, name


class Scope(dict):
    """Variables of one procedure activation; dummy scalars alias the caller."""

    def __getitem__(self, k):
        v = dict.__getitem__(self, k)
        if isinstance(v, Ref):
            return v.scope[v.name]
        return v

    def __setitem__(self, k, v):
        if k in self and isinstance(dict.__getitem__(self, k), Ref):
            r = dict.__getitem__(self, k)
            r.scope[r.name] = v
        else:
            dict.__setitem__(self, k, v)

    def bind(self, k, v):
        dict.__setitem__(self, k, v)


def f_div(a, b):
    if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
        q = abs(int(a)) // abs(int(b))
        return q if (a >= 0) == (b >= 0) else -q
    return a / b


def f_pow(a, b):
    return a ** b


def f_abs(x):
    return np.abs(x) if isinstance(x, np.ndarray) else abs(x)


def _m1(fn_s, fn_v):
    return lambda x: fn_v(x) if isinstance(x, np.ndarray) else fn_s(x)


INTRINSICS = {
    "abs": "f_abs", "sin": "f_sin", "cos": "f_cos", "exp": "f_exp", "sqrt": "f_sqrt",
    "atan": "f_atan", "real": "f_real", "dble": "f_real", "int": "f_int", "mod": "f_mod",
    "transpose": "f_transpose", "minval": "f_minval", "maxval": "f_maxval",
    "trim": "f_trim", "command_argument_count": "f_argc", "max": "f_max", "min": "f_min",
}
f_sin = _m1(math.sin, np.sin)
f_cos = _m1(math.cos, np.cos)
f_exp = _m1(math.exp, np.exp)
f_sqrt = _m1(math.sqrt, np.sqrt)
f_atan = _m1(math.atan, np.arctan)


def f_real(x, kind=None):
    return x.astype(np.float64) if isinstance(x, np.ndarray) else float(x)


def f_int(x, kind=None):
    return int(x)


def f_mod(a, b):
    return int(math.fmod(a, b)) if isinstance(a, int) else math.fmod(a, b)


def f_max(*a):
    return max(a)


def f_min(*a):
    return min(a)


def f_transpose(a):
    a2 = val(a).reshape(a.dims, order="F")
    out = FArr.zeros((a.dims[1], a.dims[0]), a.buf.dtype)
    out.flat()[:] = a2.T.reshape(-1, order="F")
    return out


def f_minval(x):
    return float(np.min(val(x)))


def f_maxval(x):
    return float(np.max(val(x)))


def f_trim(s):
    return s.rstrip()


# ---------------------------------------------------------------------------
# Formatted output (the formats the reference writes)
# ---------------------------------------------------------------------------


def _es(x, w, d):
    s = f"{x:.{d}E}"
    mant, ex = s.split("E")
    e = int(ex)
    s = f"{mant}E{'+' if e >= 0 else '-'}{abs(e):02d}"
    return s.rjust(w)


def fmt_write(fmt, items):
    fmt = fmt.strip()
    assert fmt[0] == "(" and fmt[-1] == ")", fmt
    specs = _split_top(fmt[1:-1])
    out, it = [], iter(items)
    for sp in specs:
        sp = sp.strip()
        if sp[0] in "'\"":
            out.append(sp[1:-1])
            continue
        m = re.fullmatch(r"(\d*)(a|i|es)(\d*)(?:\.(\d+))?", sp.lower())
        assert m, sp
        rep = int(m.group(1) or 1)
        for _ in range(rep):
            x = next(it)
            kind, w = m.group(2), m.group(3)
            if kind == "a":
                s = str(x)
                out.append(s.rjust(int(w)) if w else s)
            elif kind == "i":
                s = str(int(x))
                out.append(s.rjust(int(w)) if w and int(w) > 0 else s)
            else:
                out.append(_es(float(x), int(w), int(m.group(4))))
    return "".join(out)


def _split_top(s, sep=","):
    parts, depth, cur, q = [], 0, "", None
    for c in s:
        if q:
            cur += c
            if c == q:
                q = None
            continue
        if c in "'\"":
            q = c
            cur += c
            continue
        if c in "([":
            depth += 1
        elif c in ")]":
            depth -= 1
        if c == sep and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += c
    parts.append(cur)
    return parts


# ---------------------------------------------------------------------------
# Source preprocessing
# ---------------------------------------------------------------------------


def _strip_comment(line):
    q = None
    for i, c in enumerate(line):
        if q:
            if c == q:
                q = None
        elif c in "'\"":
            q = c
        elif c == "!":
            return line[:i]
    return line


def _lower_code(s):
    out, q = [], None
    for c in s:
        if q:
            out.append(c)
            if c == q:
                q = None
        elif c in "'\"":
            q = c
            out.append(c)
        else:
            out.append(c.lower())
    return "".join(out)


def statements(path):
    """Logical statements of a free-form source file (comments removed,
    continuations joined, ';' split, lower-cased outside strings)."""
    lines = open(path).read().split("\n")
    stmts, cur = [], ""
    for ln in lines:
        s = _strip_comment(ln).rstrip()
        if not s.strip():
            continue
        s = s.strip()
        if cur and s.startswith("&"):
            s = s[1:]
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        cur += s
        for part in _split_top(cur, ";"):
            if part.strip():
                stmts.append(_lower_code(part.strip()))
        cur = ""
    return stmts


# ---------------------------------------------------------------------------
# Expression parser -> Python source
# ---------------------------------------------------------------------------

TOKEN = re.compile(r"""
  (?P<ws>\s+)
| (?P<num>(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?(_[a-z0-9]+)?)
| (?P<dop>\.(and|or|not|eqv|neqv|true|false|eq|ne|lt|le|gt|ge)\.)
| (?P<str>'[^']*'|"[^"]*")
| (?P<name>[a-z_][a-z0-9_]*)
| (?P<op>\*\*|//|==|/=|<=|>=|=>|[-+*/()<>,:%\[\]=])
""", re.X)


def tokenize(s):
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN.match(s, pos)
        if not m:
            raise SyntaxError(f"cannot tokenize at: {s[pos:]!r}")
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        toks.append((kind, m.group(kind) if kind != "num" else m.group(0)))
    return toks


class ExprParser:
    """Fortran expressions to Python, fully parenthesised."""

    def __init__(self, toks, ctx):
        self.t, self.i, self.ctx = toks, 0, ctx

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else (None, None)

    def take(self, v=None):
        tok = self.t[self.i]
        if v is not None and tok[1] != v:
            raise SyntaxError(f"expected {v}, got {tok}")
        self.i += 1
        return tok

    def parse(self):
        e = self.p_or()
        return e

    def p_or(self):
        a = self.p_and()
        while self.peek()[1] == ".or.":
            self.take()
            a = f"({a} or {self.p_and()})"
        return a

    def p_and(self):
        a = self.p_not()
        while self.peek()[1] == ".and.":
            self.take()
            a = f"({a} and {self.p_not()})"
        return a

    def p_not(self):
        if self.peek()[1] == ".not.":
            self.take()
            return f"(not {self.p_not()})"
        return self.p_rel()

    RELOPS = {"==": "==", "/=": "!=", "<": "<", ">": ">", "<=": "<=", ">=": ">=",
              ".eq.": "==", ".ne.": "!=", ".lt.": "<", ".gt.": ">", ".le.": "<=",
              ".ge.": ">="}

    def p_rel(self):
        a = self.p_add()
        op = self.peek()[1]
        if op in self.RELOPS:
            self.take()
            b = self.p_add()
            return f"({a} {self.RELOPS[op]} {b})"
        return a

    def p_add(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            a = self.p_mul()
            a = f"(-{a})" if op == "-" else a
        else:
            a = self.p_mul()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            b = self.p_mul()
            a = f"({a} {op} {b})"
        return a

    def p_mul(self):
        a = self.p_pow()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            b = self.p_pow()
            a = f"({a} * {b})" if op == "*" else f"f_div({a}, {b})"
        return a

    def p_pow(self):
        a = self.p_prim()
        if self.peek()[1] == "**":
            self.take()
            b = self.p_powrhs()
            return f"f_pow({a}, {b})"
        return a

    def p_powrhs(self):
        if self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            x = self.p_pow()
            return f"(-{x})" if op == "-" else x
        return self.p_pow()

    def p_prim(self):
        kind, v = self.peek()
        if v == "(":
            self.take()
            e = self.p_or()
            self.take(")")
            return f"({e})"
        if v == "[":
            self.take()
            items = []
            while self.peek()[1] != "]":
                items.append(self.p_or())
                if self.peek()[1] == ",":
                    self.take()
            self.take("]")
            return f"f_arr([{', '.join(items)}])"
        if kind == "num":
            self.take()
            return num_literal(v)
        if kind == "str":
            self.take()
            return repr(v[1:-1])
        if kind == "dop":
            self.take()
            if v == ".true.":
                return "True"
            if v == ".false.":
                return "False"
            raise SyntaxError(v)
        if kind == "name":
            self.take()
            if self.peek()[1] == "%":
                self.take()
                comp = self.take()[1]
                return f"{self.ctx.ref(v)}.{comp}"
            if self.peek()[1] == "(":
                args = self.arglist()
                return self.ctx.apply(v, args)
            return self.ctx.ref(v)
        raise SyntaxError(f"unexpected token {v!r}")

    def arglist(self):
        """Parses '( a, b:c, :, name=x )' -> list of (keyword, python, kind)."""
        self.take("(")
        args = []
        while self.peek()[1] != ")":
            kw = None
            if self.peek()[0] == "name" and self.peek(1)[1] == "=":
                kw = self.take()[1]
                self.take("=")
            if self.peek()[1] == ":":
                self.take()
                hi = None
                if self.peek()[1] not in (",", ")"):
                    hi = self.p_or()
                args.append((kw, f"Colon(None, {hi})", "colon"))
            else:
                e = self.p_or()
                if self.peek()[1] == ":":
                    self.take()
                    hi = None
                    if self.peek()[1] not in (",", ")"):
                        hi = self.p_or()
                    args.append((kw, f"Colon({e}, {hi})", "colon"))
                else:
                    args.append((kw, e, "expr"))
            if self.peek()[1] == ",":
                self.take()
        self.take(")")
        return args


def num_literal(v):
    m = re.fullmatch(r"(\d+\.\d*|\.\d+|\d+)([ed][+-]?\d+)?(_[a-z0-9]+)?", v)
    body, ex = m.group(1), m.group(2)
    if "." not in body and ex is None:
        return str(int(body))
    s = body + (("e" + ex[1:]) if ex else "")
    return repr(float(s))


def f_arr(items):
    return np.array(items, dtype=np.float64)


# ---------------------------------------------------------------------------
# Program model
# ---------------------------------------------------------------------------


class Var:
    def __init__(self, name, typ, dims=None, intent=None, param=False, alloc=False,
                 init=None):
        self.name, self.typ, self.dims = name, typ, dims
        self.intent, self.param, self.alloc, self.init = intent, param, alloc, init


class Proc:
    def __init__(self, name, kind, args, module, result=None):
        self.name, self.kind, self.args, self.module = name, kind, args, module
        self.result = result or name
        self.vars, self.body, self.uses, self.namelists = {}, [], [], {}
        self.contains = []
        self.parent = None


class Module:
    def __init__(self, name):
        self.name = name
        self.vars, self.uses, self.procs = {}, [], []
        self.data = {}


DECL = re.compile(r"^(integer|real|logical|character|type)\b")


def parse_decl(stmt):
    """'real(rp), intent(in) :: a(n,m), b = 1' -> (typ, attrs, [(name, dims, init)])."""
    if "::" in stmt:
        head, rest = stmt.split("::", 1)
    else:
        m = re.match(r"^(integer|real\(\w+\)|real|logical)\s+(.*)$", stmt)
        head, rest = m.group(1), m.group(2)
    hp = _split_top(head)
    typ = hp[0].strip()
    attrs = [a.strip() for a in hp[1:]]
    ents = []
    for ent in _split_top(rest):
        ent = ent.strip()
        init = None
        m = re.match(r"^([a-z_][a-z0-9_]*)\s*(\(.*\))?\s*(=(?!>)\s*(.*))?$", ent)
        name, dims, init = m.group(1), m.group(2), m.group(4)
        dl = [d.strip() for d in _split_top(dims[1:-1])] if dims else None
        ents.append((name, dl, init))
    return typ, attrs, ents


def build(files):
    """Parses the source files into modules, procedures and the program."""
    mods, procs, program = {}, {}, None
    for path in files:
        st = statements(path)
        i = 0
        cur_mod, stack = None, []
        while i < len(st):
            s = st[i]
            i += 1
            m = re.match(r"^module\s+(\w+)$", s)
            if m:
                cur_mod = Module(m.group(1))
                mods[cur_mod.name] = cur_mod
                continue
            m = re.match(r"^program\s+(\w+)$", s)
            if m:
                p = Proc(m.group(1), "program", [], None)
                program = p
                procs[p.name] = p
                stack.append(p)
                continue
            if re.match(r"^end\s*(module|program)", s):
                if s.startswith("end program") or s.startswith("endprogram"):
                    stack.pop()
                else:
                    cur_mod = None
                continue
            m = re.match(r"^(?:(integer|real\(\w+\))\s+)?(subroutine|function)\s+(\w+)\s*\(([^)]*)\)\s*(?:result\((\w+)\))?$", s)
            if m:
                args = [a.strip() for a in m.group(4).split(",") if a.strip()]
                p = Proc(m.group(3), m.group(2), args, cur_mod, m.group(5))
                if m.group(1):
                    p.vars[p.result] = Var(p.result, m.group(1))
                if stack:
                    p.parent = stack[-1]
                    stack[-1].contains.append(p)
                procs[p.name] = p
                if cur_mod is not None and not stack:
                    cur_mod.procs.append(p)
                stack.append(p)
                continue
            if re.match(r"^end\s*(subroutine|function)", s):
                stack.pop()
                continue
            if s.startswith("type,") or re.match(r"^type\s+\w+$", s):
                while not re.match(r"^end\s*type", st[i]):
                    i += 1
                i += 1
                continue
            tgt = stack[-1] if stack else cur_mod
            if s in ("implicit none", "private", "contains") or s.startswith("public") \
                    or s.startswith("private"):
                continue
            m = re.match(r"^use\s*(?:,\s*intrinsic\s*::)?\s*(\w+)\s*(?:,\s*only\s*:\s*(.*))?$", s)
            if m:
                names = None
                if m.group(2) is not None:
                    names = []
                    for it in m.group(2).split(","):
                        it = it.strip()
                        if "=>" in it:
                            local, remote = [x.strip() for x in it.split("=>")]
                        else:
                            local = remote = it
                        names.append((local, remote))
                tgt.uses.append((m.group(1), names))
                continue
            m = re.match(r"^namelist\s*/(\w+)/\s*(.*)$", s)
            if m:
                tgt.namelists[m.group(1)] = [x.strip() for x in m.group(2).split(",")]
                continue
            if DECL.match(s) and ("::" in s or re.match(r"^(integer|real\(\w+\)|real|logical)\s+[a-z]", s)) \
                    and not re.match(r"^(integer|real)\s*(\(\w+\))?\s*function", s):
                typ, attrs, ents = parse_decl(s)
                intent = None
                for a in attrs:
                    mm = re.match(r"intent\((\w+)\)", a)
                    if mm:
                        intent = mm.group(1)
                for name, dims, init in ents:
                    tgt.vars[name] = Var(name, typ, dims, intent, "parameter" in attrs,
                                         "allocatable" in attrs, init)
                continue
            tgt.body.append(s)
    return mods, procs, program


# ---------------------------------------------------------------------------
# Code generation
# ---------------------------------------------------------------------------


class Ctx:
    """Name resolution of one procedure (or module initialiser)."""

    def __init__(self, interp, proc=None, module=None):
        self.I, self.proc, self.module = interp, proc, module

    def owner(self, name):
        """Where `name` lives: ('V', proc) local, ('M', modname), ('H', host proc)."""
        p = self.proc
        if p is not None:
            if name in p.vars or name in p.args:
                return ("V", None)
            host = p.parent
            while host is not None:
                if name in host.vars:
                    return ("H", host.name)
                for mod, names in host.uses:
                    r = self.I.resolve_use(mod, names, name)
                    if r:
                        return r
                host = host.parent
            for mod, names in p.uses:
                r = self.I.resolve_use(mod, names, name)
                if r:
                    return r
        mod = self.module
        if mod is not None:
            if name in mod.vars:
                return ("M", mod.name, name)
            for m2, names in mod.uses:
                r = self.I.resolve_use(m2, names, name)
                if r:
                    return r
        return None

    def ref(self, name):
        o = self.owner(name)
        if o is None:
            raise NameError(f"unresolved name {name} in {self.proc.name if self.proc else '?'}")
        if o[0] == "V":
            return f"V[{name!r}]"
        if o[0] == "H":
            return f"H[{o[1]!r}][{name!r}]"
        return f"MOD[{o[1]!r}][{o[2]!r}]"

    def var(self, name):
        o = self.owner(name)
        if o is None:
            return None
        if o[0] == "V":
            return self.proc.vars.get(name)
        if o[0] == "H":
            return self.I.procs[o[1]].vars.get(name)
        return self.I.mods[o[1]].vars.get(o[2])

    def is_array(self, name):
        v = self.var(name)
        return v is not None and (v.dims is not None or v.alloc)

    def apply(self, name, args):
        if self.owner(name) is not None and self.is_array(name):
            idx = ", ".join(a[1] for a in args)
            return f"{self.ref(name)}.get({idx})"
        if name in INTRINSICS:
            pos = [a[1] for a in args if a[0] is None]
            return f"{INTRINSICS[name]}({', '.join(pos)})"
        p = self.I.proc_for(name, self)
        if p is None:
            raise NameError(f"unknown function {name}")
        return f"CALL({p.name!r}, [{', '.join('(lambda: ' + a[1] + ')' for a in args)}], None)"


class Interp:
    def __init__(self, files, cwd, argv=()):
        self.mods, self.procs, self.program = build(files)
        # The intrinsic module iso_fortran_env: kind numbers and units.
        iso = Module("iso_fortran_env")
        for name, value in (("int64", 8), ("real64", 8), ("int32", 4),
                            ("error_unit", 0), ("output_unit", 6)):
            iso.vars[name] = Var(name, "integer", init=str(value), param=True)
        self.mods = {"iso_fortran_env": iso, **self.mods}
        self.cwd, self.argv = cwd, list(argv)
        self.MOD = {m: Scope() for m in self.mods}
        self.HOST = {}
        self.out = []
        self.units = {}
        self.compiled = {}
        self.env = {k: v for k, v in globals().items()}
        self.env.update(MOD=self.MOD, H=self.HOST, CALL=self.call, IO=self, f_argc=self.argc)
        for m in self.mods.values():
            self._init_module(m)

    # -- name resolution helpers --
    def resolve_use(self, mod, names, name):
        if mod not in self.mods:
            return None
        if names is None:
            if name in self.mods[mod].vars:
                return ("M", mod, name)
            for m2, n2 in self.mods[mod].uses:
                r = self.resolve_use(m2, n2, name)
                if r:
                    return r
            return None
        for local, remote in names:
            if local == name:
                if remote in self.mods[mod].vars:
                    return ("M", mod, remote)
                for m2, n2 in self.mods[mod].uses:
                    r = self.resolve_use(m2, n2, remote)
                    if r:
                        return r
        return None

    def proc_for(self, name, ctx):
        return self.procs.get(name)

    def _init_module(self, m):
        ctx = Ctx(self, None, m)
        for v in m.vars.values():
            self.MOD[m.name][v.name] = self._initial(v, ctx, None)

    def _initial(self, v, ctx, scope):
        if v.typ.startswith("type"):
            return TimerStub()
        if v.alloc:
            return None
        if v.init is not None:
            code = ExprParser(tokenize(v.init), ctx).parse()
            x = eval(code, self.env, {"V": scope})
            if v.dims and not isinstance(x, FArr):
                a = FArr.zeros([len(np.atleast_1d(x))], np.float64)
                a.flat()[:] = x
                return a
            if v.typ.startswith("real") and isinstance(x, int):
                return float(x)
            return x
        if v.typ.startswith("character"):
            return ""
        if v.typ.startswith("logical"):
            return False
        return 0 if v.typ.startswith("integer") else 0.0

    def argc(self):
        return len(self.argv)

    # -- procedure execution --
    def compile(self, p):
        if p.name in self.compiled:
            return self.compiled[p.name]
        ctx = Ctx(self, p, p.module if p.module else self._module_of(p))
        lines = ["def _proc(V):"]
        gen = StmtGen(ctx, lines)
        gen.block(p.body, 1)
        lines.append("    return None")
        src = "\n".join(lines)
        ns = {}
        exec(compile(src, f"<f90:{p.name}>", "exec"), self.env, ns)
        self.compiled[p.name] = (ns["_proc"], ctx)
        return self.compiled[p.name]

    def _module_of(self, p):
        while p.parent is not None:
            p = p.parent
        return p.module

    def call(self, name, thunks, refs):
        """Calls procedure `name` with actual arguments.  thunks evaluate each
        actual; refs[i] (if given) is a (kind, payload) describing how the
        actual can be passed by reference."""
        if name in STUBS:
            return STUBS[name](self, thunks, refs)
        p = self.procs[name]
        fn, ctx = self.compile(p)
        V = Scope()
        # scalars and arrays of the dummies
        for k, dummy in enumerate(p.args):
            r = refs[k] if refs else None
            if r is not None and r[0] == "scalar":
                V.bind(dummy, Ref(r[1], r[2]))
            elif r is not None and r[0] == "array" and r[1] is not None:
                V.bind(dummy, r[1])
            else:
                x = thunks[k]()
                V.bind(dummy, x)
        # declared locals and reshaped dummies
        for v in p.vars.values():
            if v.name in p.args:
                if v.dims is not None:
                    dims = [eval(ExprParser(tokenize(d), ctx).parse(), self.env, {"V": V})
                            for d in v.dims]
                    a = dict.__getitem__(V, v.name)
                    if isinstance(a, FArr):
                        V.bind(v.name, a.view(dims))
                    else:
                        arr = FArr.zeros(dims, np.float64)
                        arr.flat()[:] = a
                        V.bind(v.name, arr)
                continue
            if v.dims is not None and not v.alloc:
                dims = [eval(ExprParser(tokenize(d), ctx).parse(), self.env, {"V": V})
                        for d in v.dims]
                dt = np.int64 if v.typ.startswith("integer") else np.float64
                if v.param and v.init is not None:
                    V.bind(v.name, self._initial(v, ctx, V))
                else:
                    V.bind(v.name, FArr.zeros(dims, dt))
            else:
                V.bind(v.name, self._initial(v, ctx, V))
        if p.kind == "program" or p.contains:
            self.HOST[p.name] = V
        fn(V)
        if p.kind == "function":
            return V[p.result]
        return None

    # -- I/O --
    def open(self, unit, fname):
        self.units[unit] = {"lines": open(os.path.join(self.cwd, fname)).read().split("\n"),
                            "pos": 0, "name": fname}

    def read_list(self, unit, targets):
        u = self.units[unit]
        need = sum(t.size if isinstance(t, FArr) else 1 for t in targets)
        vals = []
        while len(vals) < need:
            vals.extend(u["lines"][u["pos"]].replace(",", " ").split())
            u["pos"] += 1
        vals = vals[:need]
        k = 0
        for t in targets:
            if isinstance(t, FArr):
                t.flat()[:] = [float(x.replace("d", "e").replace("D", "E"))
                               for x in vals[k:k + t.size]]
                k += t.size
        return vals

    def read_namelist(self, unit, group, scope_setter):
        text = "\n".join(self.units[unit]["lines"])
        body = []
        for ln in text.split("\n"):
            body.append(_strip_comment(ln))
        text = "\n".join(body)
        m = re.search(r"&" + group + r"\b(.*?)/", text, re.I | re.S)
        if not m:
            raise FortranStop(f"namelist {group} not found")
        for item in _split_top(m.group(1).replace("\n", ","), ","):
            item = item.strip()
            if not item:
                continue
            k, v = [x.strip() for x in item.split("=", 1)]
            scope_setter(k.lower(), v)

    def close(self, unit):
        self.units.pop(unit, None)


class TimerStub:
    count_start = 0
    count_accum = 0
    count_rate = 1


def _stub_timer(interp, thunks, refs):
    return None


def _stub_elapsed(interp, thunks, refs):
    return 0.0


STUBS = {"timer_start": _stub_timer, "timer_stop": _stub_timer,
         "timer_elapsed": _stub_elapsed, "flush": _stub_timer,
         "system_clock": _stub_timer}


def _nml_value(v, cur):
    v = v.strip()
    if v[:1] in "'\"":
        return v[1:-1]
    if isinstance(cur, int) and not isinstance(cur, bool):
        return int(v)
    return float(v.lower().replace("d", "e"))


class StmtGen:
    def __init__(self, ctx, lines):
        self.ctx, self.lines = ctx, lines
        self.tmp = 0

    def emit(self, ind, s):
        self.lines.append("    " * ind + s)

    def expr(self, s):
        return ExprParser(tokenize(s), self.ctx).parse()

    def block(self, body, ind):
        i = 0
        n0 = len(self.lines)
        while i < len(body):
            i = self.stmt(body, i, ind)
        if len(self.lines) == n0:
            self.emit(ind, "pass")

    def _find_end(self, body, i, opener, closer, mids=()):
        depth, j, marks = 0, i, []
        while j < len(body):
            s = body[j]
            if opener(s):
                depth += 1
            elif closer(s):
                depth -= 1
                if depth == 0:
                    return j, marks
            elif depth == 1 and any(m(s) for m in mids):
                marks.append(j)
            j += 1
        raise SyntaxError("unterminated block")

    def stmt(self, body, i, ind):
        s = body[i]
        # do loop
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", s)
        if m:
            end, _ = self._find_end(body, i, lambda x: re.match(r"^do\b", x) is not None,
                                    lambda x: re.match(r"^end\s*do$", x) is not None)
            bounds = _split_top(m.group(2))
            lo, hi = self.expr(bounds[0]), self.expr(bounds[1])
            st = self.expr(bounds[2]) if len(bounds) > 2 else "1"
            var = self.ctx.ref(m.group(1))
            it = f"_it{self.tmp}"
            self.tmp += 1
            self.emit(ind, f"for {it} in range(int({lo}), int({hi}) + (1 if {st} > 0 else -1), int({st})):")
            self.emit(ind + 1, f"{var} = {it}")
            self.block(body[i + 1:end], ind + 1)
            return end + 1
        # block if
        m = re.match(r"^if\s*\((.*)\)\s*then$", s)
        if m:
            end, marks = self._find_end(
                body, i, lambda x: re.match(r"^if\s*\(.*\)\s*then$", x) is not None,
                lambda x: re.match(r"^end\s*if$", x) is not None,
                (lambda x: re.match(r"^else", x) is not None,))
            self.emit(ind, f"if {self.expr(m.group(1))}:")
            segs = [i] + marks + [end]
            for k in range(len(segs) - 1):
                if k > 0:
                    hdr = body[segs[k]]
                    mm = re.match(r"^else\s*if\s*\((.*)\)\s*then$", hdr)
                    if mm:
                        self.emit(ind, f"elif {self.expr(mm.group(1))}:")
                    else:
                        self.emit(ind, "else:")
                self.block(body[segs[k] + 1:segs[k + 1]], ind + 1)
            return end + 1
        # select case
        m = re.match(r"^select\s*case\s*\((.*)\)$", s)
        if m:
            end, marks = self._find_end(
                body, i, lambda x: x.startswith("select"),
                lambda x: re.match(r"^end\s*select$", x) is not None,
                (lambda x: re.match(r"^case\b", x) is not None,))
            t = f"_sel{self.tmp}"
            self.tmp += 1
            self.emit(ind, f"{t} = {self.expr(m.group(1))}")
            first = True
            segs = marks + [end]
            for k in range(len(segs) - 1):
                hdr = body[segs[k]]
                if re.match(r"^case\s+default$", hdr):
                    self.emit(ind, "else:" if not first else "if True:")
                else:
                    mm = re.match(r"^case\s*\((.*)\)$", hdr)
                    vals = [self.expr(x) for x in _split_top(mm.group(1))]
                    cond = " or ".join(f"{t} == {v}" for v in vals)
                    self.emit(ind, f"{'if' if first else 'elif'} {cond}:")
                first = False
                self.block(body[segs[k] + 1:segs[k + 1]], ind + 1)
            return end + 1
        # one-line if
        m = re.match(r"^if\s*\((.*)\)\s*(\w.*)$", s)
        if m and not s.endswith("then"):
            cond, rest = self._split_if(s)
            self.emit(ind, f"if {self.expr(cond)}:")
            self.stmt([rest], 0, ind + 1)
            return i + 1
        self.simple(s, ind)
        return i + 1

    def _split_if(self, s):
        depth = 0
        start = s.index("(")
        for j in range(start, len(s)):
            if s[j] == "(":
                depth += 1
            elif s[j] == ")":
                depth -= 1
                if depth == 0:
                    return s[start + 1:j], s[j + 1:].strip()
        raise SyntaxError(s)

    def simple(self, s, ind):
        if s == "return":
            self.emit(ind, "return None")
            return
        if s.startswith("error stop"):
            self.emit(ind, f"raise FortranStop({s!r})")
            return
        m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", s)
        if m:
            self.emit_call(m.group(1), m.group(3) or "", ind)
            return
        m = re.match(r"^allocate\s*\((.*)\)$", s)
        if m:
            for ent in _split_top(m.group(1)):
                mm = re.match(r"^\s*(\w+)\s*\((.*)\)\s*$", ent)
                name = mm.group(1)
                dims = ", ".join(self.expr(d) for d in _split_top(mm.group(2)))
                v = self.ctx.var(name)
                dt = "np.int64" if v.typ.startswith("integer") else "np.float64"
                self.emit(ind, f"{self.ctx.ref(name)} = FArr.zeros([{dims}], {dt})")
            return
        m = re.match(r"^open\s*\((.*)\)$", s)
        if m:
            parts = _split_top(m.group(1))
            unit = self.expr(parts[0])
            fname = None
            for p in parts[1:]:
                k, v = p.split("=", 1)
                if k.strip() == "file":
                    fname = self.expr(v)
            self.emit(ind, f"IO.open({unit}, {fname})")
            return
        m = re.match(r"^close\s*\((.*)\)$", s)
        if m:
            self.emit(ind, f"IO.close({self.expr(_split_top(m.group(1))[0])})")
            return
        m = _io_stmt("read", s)
        if m:
            ctl = _split_top(m.group(1))
            unit = self.expr(ctl[0])
            if len(ctl) > 1 and ctl[1].strip().startswith("nml"):
                grp = ctl[1].split("=", 1)[1].strip()
                names = self._namelist(grp)
                setter = f"_nml{self.tmp}"
                self.tmp += 1
                self.emit(ind, f"def {setter}(k, v):")
                for nm in names:
                    self.emit(ind + 1, f"if k == {nm!r}: {self.ctx.ref(nm)} = _nml_value(v, {self.ctx.ref(nm)})")
                self.emit(ind, f"IO.read_namelist({unit}, {grp!r}, {setter})")
                return
            tg = ", ".join(self.ctx.ref(t.strip()) for t in _split_top(m.group(2)))
            self.emit(ind, f"IO.read_list({unit}, [{tg}])")
            return
        m = _io_stmt("write", s)
        if m:
            ctl = _split_top(m.group(1))
            fmt = ctl[1].strip() if len(ctl) > 1 else "*"
            items = ", ".join(self.expr(x) for x in _split_top(m.group(2))) if m.group(2) else ""
            fmt_py = self.expr(fmt) if fmt != "*" else "None"
            target = ctl[0].strip()
            if target == "*" or re.fullmatch(r"\d+|error_unit", target):
                self.emit(ind, f"IO.out.append(fmt_write({fmt_py}, [{items}]) if {fmt_py} else ' '.join(map(str, [{items}])))")
            else:
                self.emit(ind, f"{self.ctx.ref(target)} = fmt_write({fmt_py}, [{items}])")
            return
        if s.startswith("flush"):
            return
        # assignment
        lhs, rhs = self._split_assign(s)
        r = self.expr(rhs)
        m = re.match(r"^(\w+)\s*%\s*(\w+)$", lhs)
        if m:
            self.emit(ind, f"{self.ctx.ref(m.group(1))}.{m.group(2)} = {r}")
            return
        m = re.match(r"^(\w+)\s*(\((.*)\))?$", lhs)
        name = m.group(1)
        if m.group(2):
            p = ExprParser(tokenize(m.group(2)), self.ctx)
            args = p.arglist()
            idx = ", ".join(a[1] for a in args)
            self.emit(ind, f"{self.ctx.ref(name)}.set({r}, {idx})")
        elif self.ctx.is_array(name):
            self.emit(ind, f"{self.ctx.ref(name)}.set({r})")
        else:
            v = self.ctx.var(name)
            if v is not None and v.typ.startswith("real"):
                self.emit(ind, f"{self.ctx.ref(name)} = f_real({r})")
            else:
                self.emit(ind, f"{self.ctx.ref(name)} = {r}")

    def _namelist(self, grp):
        p = self.ctx.proc
        while p is not None:
            if grp in p.namelists:
                return p.namelists[grp]
            p = p.parent
        raise NameError(grp)

    def _split_assign(self, s):
        depth = 0
        for j, c in enumerate(s):
            if c in "([":
                depth += 1
            elif c in ")]":
                depth -= 1
            elif c == "=" and depth == 0 and s[j + 1:j + 2] != "=" and s[j - 1] not in "<>/=":
                return s[:j].strip(), s[j + 1:].strip()
        raise SyntaxError(f"not an assignment: {s}")

    def emit_call(self, name, argstr, ind):
        if name in ("system_clock", "flush"):
            return
        if name == "get_command_argument":
            a = _split_top(argstr)
            self.emit(ind, f"{self.ctx.ref(a[1].strip())} = IO.argv[{self.expr(a[0])} - 1]")
            return
        args = _split_top(argstr) if argstr.strip() else []
        thunks, refs = [], []
        for a in args:
            a = a.strip()
            e = self.expr(a)
            thunks.append(f"(lambda: {e})")
            m = re.fullmatch(r"(\w+)", a)
            if m and self.ctx.owner(a) is not None:
                if self.ctx.is_array(a):
                    refs.append(f"('array', {self.ctx.ref(a)})")
                else:
                    o = self.ctx.owner(a)
                    scope = ("V" if o[0] == "V" else
                             f"H[{o[1]!r}]" if o[0] == "H" else f"MOD[{o[1]!r}]")
                    nm = a if o[0] != "M" else o[2]
                    refs.append(f"('scalar', {scope}, {nm!r})")
                continue
            m = re.fullmatch(r"(\w+)\s*\((.*)\)", a)
            if m and self.ctx.owner(m.group(1)) is not None and self.ctx.is_array(m.group(1)):
                p = ExprParser(tokenize("(" + m.group(2) + ")"), self.ctx)
                idx = ", ".join(x[1] for x in p.arglist())
                refs.append(f"('array', {self.ctx.ref(m.group(1))}.section_view(({idx},)))")
                continue
            refs.append("None")
        self.emit(ind, f"CALL({name!r}, [{', '.join(thunks)}], [{', '.join(refs)}])")


class _IOMatch:
    def __init__(self, ctl, items):
        self._g = (None, ctl, items)

    def group(self, k):
        return self._g[k]


def _io_stmt(kw, s):
    """Splits 'read(ctl) items' / 'write(ctl) items' with quote-aware
    parenthesis matching (formats contain parentheses)."""
    m = re.match(r"^" + kw + r"\s*\(", s)
    if not m:
        return None
    depth, q = 0, None
    for j in range(m.end() - 1, len(s)):
        c = s[j]
        if q:
            if c == q:
                q = None
            continue
        if c in "'\"":
            q = c
        elif c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
            if depth == 0:
                return _IOMatch(s[m.end():j], s[j + 1:].strip())
    raise SyntaxError(s)


def run_program(interp):
    """Runs the main program unit."""
    interp.call(interp.program.name, [], [])
    return interp.out
