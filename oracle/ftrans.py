"""Restricted Fortran 90 -> C translator for PICSAR's hot-path routines.

TEST INFRASTRUCTURE ONLY.  The image has no Fortran compiler, so the
reference's own routines cannot be built as they are.  This script reads the
reference Fortran sources where they lie and emits C that follows their
statements one for one:

* the same loops, loop bounds (trip count fixed at loop entry, as Fortran
  does), branches and operation order (left-to-right evaluation,
  parenthesisation kept);
* the same types: REAL(num) -> double, default REAL literals -> float (so a
  default-real subexpression rounds as Fortran does), INTEGER(idp) ->
  int64_t, INTEGER(isp)/INTEGER -> int32_t, LOGICAL(lp) -> int64_t;
* Fortran intrinsic semantics: FLOOR/NINT/INT return default INTEGER,
  NINT rounds half away from zero (lround), x**2 -> x*x;
* arrays column-major with their declared lower bounds, dummies passed by
  reference, whole-array assignments expanded to element loops;
* module variables (clight, dt, particle_pusher) become globals set through
  ``pxrref_set_module``.

The output (``oracle/_ref/pxr_ref.c``) is compiled with ``-O2
-ffp-contract=off`` into ``oracle/_ref/libpxr_ref.so`` by the ``ref`` target
of ``oracle/Makefile``; the oracle is then checked bit-for-bit against the
reference's code run this way (``tests/test_oracle_vs_reference.py``).
Nothing of the reference's text is kept in the repository: the C is generated
into the git-ignored ``oracle/_ref/``.

Only the subset of Fortran used by the routines in ``ROUTINES`` is handled;
anything else raises ``FtransError`` naming the construct.

Usage: python oracle/ftrans.py <picsar src dir> <out.c>
"""
from __future__ import annotations

import os
import re
import sys

# (file under src/, routine names) of the reference hot path.
ROUTINES = [
    ("particle_pushers/boris_pusher/boris_3d.F90",
     ["pxr_boris_push_u_3d", "pxr_set_gamma", "pxr_pushxyz"]),
    ("particle_pushers/vay_pusher/vay_3d.F90", ["pxr_ebcancelpush3d"]),
    ("particle_pushers/particle_pusher_manager_3d.F90",
     [f"field_gathering_plus_particle_pusher_{o}_{o}_{o}" for o in (1, 2, 3)]),
    ("particle_deposition/current_deposition/esirkepov/esirkepov_3d.F90",
     [f"depose_jxjyjz_esirkepov_{o}_{o}_{o}" for o in (1, 2, 3)]
     + ["pxr_depose_jxjyjz_esirkepov_n"]),
    ("field_solvers/Maxwell/yee_solver/yee.F90",
     ["pxrpush_em3d_evec", "pxrpush_em3d_bvec", "pxrpush_em3d_evec_norder",
      "pxrpush_em3d_bvec_norder", "pxrpush_em2d_evec", "pxrpush_em2d_bvec"]),
    ("submain.F90", ["FD_weights"]),
    ("field_gathering/energy_conserving/field_gathering_o1_2d.F90",
     ["pxr_gete2dxz_energy_conserving_scalar_1_1", "pxr_getb2dxz_energy_conserving_scalar_1_1"]),
    ("field_gathering/energy_conserving/field_gathering_o2_2d.F90",
     ["pxr_gete2dxz_energy_conserving_scalar_2_2", "pxr_getb2dxz_energy_conserving_scalar_2_2"]),
    ("field_gathering/energy_conserving/field_gathering_o3_2d.F90",
     ["pxr_gete2dxz_energy_conserving_scalar_3_3", "pxr_getb2dxz_energy_conserving_scalar_3_3"]),
    ("particle_deposition/current_deposition/esirkepov/esirkepov_2d.F90",
     [f"pxr_depose_jxjyjz_esirkepov2d_{o}_{o}" for o in (1, 2, 3)]),
    ("particle_pushers/boris_pusher/boris_2d.F90", ["pxr_pushxz"]),
    ("field_gathering/energy_conserving/field_gathering_o1_3d.F90",
     ["gete3d_energy_conserving_scalar_1_1_1", "getb3d_energy_conserving_scalar_1_1_1"]),
    ("field_gathering/energy_conserving/field_gathering_o2_3d.F90",
     ["gete3d_energy_conserving_scalar_2_2_2", "getb3d_energy_conserving_scalar_2_2_2"]),
    ("field_gathering/energy_conserving/field_gathering_o3_3d.F90",
     ["gete3d_energy_conserving_scalar_3_3_3", "getb3d_energy_conserving_scalar_3_3_3"]),
    ("particle_deposition/charge_deposition/charge_deposition_3d.F90",
     [f"depose_rho_scalar_{o}_{o}_{o}" for o in (1, 2, 3)]),
]

# module variables the routines take by USE association
MODULE_VARS = {"clight": "double", "dt": "double", "particle_pusher": "int64_t",
               "mu0": "double", "eps0": "double"}

CTYPE_RANK = {"bool": 0, "int32_t": 1, "int64_t": 2, "float": 3, "double": 4}


class FtransError(Exception):
    pass


# ---------------------------------------------------------------------------
# Source handling: preprocessor, comments, continuations
# ---------------------------------------------------------------------------
def _pp_eval(expr, defined):
    """Evaluate a #if expression with every macro undefined unless listed."""
    e = expr
    e = re.sub(r"defined\s*\(\s*(\w+)\s*\)", lambda m: "1" if m.group(1) in defined else "0", e)
    e = re.sub(r"defined\s+(\w+)", lambda m: "1" if m.group(1) in defined else "0", e)
    e = re.sub(r"\b[A-Za-z_]\w*\b", "0", e)
    e = e.replace("&&", " and ").replace("||", " or ")
    e = re.sub(r"!(?!=)", " not ", e)
    return bool(eval(e, {}, {}))


def preprocess(lines, defined=()):
    out = []
    stack = []  # (active, taken)
    active = True
    for ln, line in lines:
        s = line.strip()
        if s.startswith("#"):
            d = s[1:].strip()
            word = d.split(None, 1)[0] if d else ""
            rest = d[len(word):].strip()
            if word == "if":
                v = _pp_eval(rest, defined)
                stack.append((active, v))
                active = active and v
            elif word == "ifdef":
                v = rest.split()[0] in defined
                stack.append((active, v))
                active = active and v
            elif word == "ifndef":
                v = rest.split()[0] not in defined
                stack.append((active, v))
                active = active and v
            elif word == "elif":
                parent, taken = stack[-1]
                v = (not taken) and _pp_eval(rest, defined)
                stack[-1] = (parent, taken or v)
                active = parent and v
            elif word == "else":
                parent, taken = stack[-1]
                stack[-1] = (parent, True)
                active = parent and not taken
            elif word == "endif":
                parent, _ = stack.pop()
                active = parent
            continue
        if active:
            out.append((ln, line))
    return out


def _strip_comment(s):
    q = None
    for i, c in enumerate(s):
        if q:
            if c == q:
                q = None
        elif c in "'\"":
            q = c
        elif c == "!":
            return s[:i]
    return s


def logical_lines(lines):
    """Join continuation lines and split on ';' -> list of (line, text)."""
    out = []
    buf, start = "", None
    for ln, line in lines:
        s = _strip_comment(line).rstrip()
        if not s.strip():
            continue
        t = s.strip()
        if buf and t.startswith("&"):
            t = t[1:]
        if start is None:
            start = ln
        if t.endswith("&"):
            buf += t[:-1] + " "
            continue
        buf += t
        for part in buf.split(";"):
            if part.strip():
                out.append((start, part.strip()))
        buf, start = "", None
    return out


def extract_routine(path, name):
    with open(path) as f:
        raw = [(i + 1, l.rstrip("\n")) for i, l in enumerate(f)]
    st = None
    for i, (ln, l) in enumerate(raw):
        if re.match(r"\s*SUBROUTINE\s+" + re.escape(name) + r"\s*\(", l, re.I):
            st = i
            break
    if st is None:
        raise FtransError(f"{name} not found in {path}")
    for j in range(st, len(raw)):
        if re.match(r"\s*END\s+SUBROUTINE\b", raw[j][1], re.I):
            return raw[st:j + 1]
    raise FtransError(f"end of {name} not found")


# ---------------------------------------------------------------------------
# Expressions
# ---------------------------------------------------------------------------
_TOK = re.compile(r"""
  (?P<num>(\d+\.\d*|\.\d+|\d+)([edED][+-]?\d+)?(_\w+)?)
 |(?P<dot>\.(and|or|not|eq|ne|lt|gt|le|ge|true|false|eqv|neqv)\.)
 |(?P<name>[A-Za-z_]\w*)
 |(?P<op>\*\*|==|/=|<=|>=|<|>|[-+*/(),:=%])
 |(?P<ws>\s+)
""", re.X | re.I)


def tokenize(s):
    toks, i = [], 0
    while i < len(s):
        m = _TOK.match(s, i)
        if not m:
            raise FtransError(f"cannot tokenize: {s[i:]!r}")
        i = m.end()
        k = m.lastgroup
        if k == "ws":
            continue
        v = m.group(k)
        if k == "dot":
            v = v.lower()
        elif k == "name":
            v = v.lower()
        toks.append((k, v))
    return toks


class P:
    """Pratt parser over one token list."""

    BIN = {".or.": 1, ".and.": 2, "==": 4, "/=": 4, "<": 4, ">": 4, "<=": 4, ">=": 4,
           ".eq.": 4, ".ne.": 4, ".lt.": 4, ".gt.": 4, ".le.": 4, ".ge.": 4,
           "+": 5, "-": 5, "*": 6, "/": 6, "**": 7}

    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else (None, None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, v):
        k, x = self.next()
        if x != v:
            raise FtransError(f"expected {v!r}, got {x!r}")

    def at_end(self):
        return self.i >= len(self.t)

    def expr(self, minp=1):
        k, v = self.peek()
        if v in ("-", "+"):
            self.next()
            x = self.expr(6)
            left = ("un", v, x)
        elif v == ".not.":
            self.next()
            left = ("un", "!", self.expr(3))
        else:
            left = self.primary()
        while True:
            k, v = self.peek()
            if v not in self.BIN:
                break
            p = self.BIN[v]
            if p < minp:
                break
            self.next()
            if v == "**":
                right = self.expr(p)          # right associative
            else:
                right = self.expr(p + 1)
            left = ("bin", v, left, right)
        return left

    def primary(self):
        k, v = self.next()
        if k == "num":
            return ("num", v)
        if k == "dot":
            if v in (".true.", ".false."):
                return ("bool", v == ".true.")
            raise FtransError(f"unexpected {v}")
        if v == "(":
            e = self.expr()
            self.expect(")")
            return ("paren", e)
        if k == "name":
            if self.peek()[1] == "(":
                self.next()
                args = []
                if self.peek()[1] != ")":
                    while True:
                        args.append(self.arg())
                        if self.peek()[1] == ",":
                            self.next()
                            continue
                        break
                self.expect(")")
                return ("ref", v, args)
            return ("name", v)
        raise FtransError(f"unexpected token {v!r}")

    def arg(self):
        # lo:hi section, keyword arg, or expression
        if self.peek()[1] == ":":
            self.next()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("range", None, hi)
        k, v = self.peek()
        if k == "name" and self.i + 1 < len(self.t) and self.t[self.i + 1][1] == "=":
            self.next()
            self.next()
            return ("kw", v, self.expr())
        e = self.expr()
        if self.peek()[1] == ":":
            self.next()
            hi = None if self.peek()[1] in (",", ")") else self.expr()
            return ("range", e, hi)
        return e


def parse_expr(s):
    p = P(tokenize(s))
    e = p.expr()
    if not p.at_end():
        raise FtransError(f"trailing tokens in {s!r}")
    return e


def split_top(s, sep=","):
    out, depth, cur = [], 0, ""
    for c in s:
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c == sep and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += c
    out.append(cur)
    return [x.strip() for x in out]


# ---------------------------------------------------------------------------
# Routine translation
# ---------------------------------------------------------------------------
KINDS = {"num": "double", "8": None, "idp": "int64_t", "isp": "int32_t", "lp": "int64_t",
         "4": None}


def _ctype(base, kind):
    base = base.lower()
    if base == "real":
        if kind in (None, "4"):
            return "float"
        return "double"
    if base == "integer":
        if kind in ("idp", "8"):
            return "int64_t"
        return "int32_t"
    if base == "logical":
        if kind in ("lp", "8"):
            return "int64_t"
        return "int32_t"
    raise FtransError(f"type {base}")


class Var:
    def __init__(self, name, ctype):
        self.name, self.ctype = name, ctype
        self.dims = None          # list of (lo_expr_ast, hi_expr_ast) or None
        self.dummy = False
        self.param = None         # init expression for PARAMETER
        self.alloc = False


class Routine:
    def __init__(self, name, lines, src, known):
        self.name = name
        self.src = src
        self.known = known        # other routine names -> Routine (for CALL)
        self.vars = {}
        self.args = []
        self.uses = set()
        self.body = []
        self.tmp = 0
        self._parse(lines)

    # -- declarations ------------------------------------------------------
    def _parse(self, lines):
        ll = logical_lines(lines)
        ln, head = ll[0]
        m = re.match(r"subroutine\s+(\w+)\s*\((.*)\)\s*$", head, re.I)
        if not m:
            raise FtransError(f"bad header {head}")
        self.args = [a.strip().lower() for a in m.group(2).split(",") if a.strip()]
        stmts = ll[1:]
        i = 0
        for ln, s in stmts:
            low = s.lower()
            if low.startswith("use "):
                mm = re.match(r"use\s+\w+\s*,\s*only\s*:\s*(.*)$", low)
                if mm:
                    for n in mm.group(1).split(","):
                        n = n.strip()
                        if n in MODULE_VARS:
                            self.uses.add(n)
                continue
            if low.startswith("implicit"):
                continue
            if re.match(r"(real|integer|logical)\b", low) and "::" in s:
                self._decl(s)
                continue
            self.body.append((ln, s))
        for a in self.args:
            if a not in self.vars:
                raise FtransError(f"{self.name}: undeclared dummy {a}")
            self.vars[a].dummy = True

    def _decl(self, s):
        spec, ents = s.split("::", 1)
        parts = split_top(spec)
        m = re.match(r"(real|integer|logical)\s*(\((.*)\))?$", parts[0], re.I)
        if not m:
            raise FtransError(f"type spec {parts[0]}")
        kind = m.group(3)
        if kind:
            kind = kind.lower().replace("kind", "").replace("=", "").strip()
        ctype = _ctype(m.group(1), kind)
        dims, param, alloc = None, False, False
        for a in parts[1:]:
            al = a.lower()
            if al.startswith("dimension"):
                dims = self._dims(a[a.index("(") + 1:a.rindex(")")])
            elif al == "parameter":
                param = True
            elif al == "allocatable":
                alloc = True
            elif al.startswith("intent") or al in ("target", "save"):
                pass
            else:
                raise FtransError(f"attribute {a}")
        for e in split_top(ents):
            init = None
            if "=" in e and not re.search(r"[<>/=]=", e):
                e, init = e.split("=", 1)
                e = e.strip()
            mm = re.match(r"(\w+)\s*(\((.*)\))?$", e.strip())
            nm = mm.group(1).lower()
            v = Var(nm, ctype)
            v.dims = self._dims(mm.group(3)) if mm.group(3) else dims
            v.alloc = alloc
            if param:
                v.param = parse_expr(init)
            self.vars[nm] = v

    def _dims(self, s):
        out = []
        for d in split_top(s):
            if d == ":":
                out.append((None, None))
            elif ":" in split_top(d, ":")[0] or len(split_top(d, ":")) == 2:
                lo, hi = split_top(d, ":")
                out.append((parse_expr(lo), parse_expr(hi)))
            else:
                out.append((("num", "1"), parse_expr(d)))
        return out

    # -- expressions -------------------------------------------------------
    def lookup(self, n):
        if n in self.vars:
            return self.vars[n]
        return None

    def scalar_ref(self, n):
        v = self.lookup(n)
        if v is None:
            if n in self.uses or n in MODULE_VARS:
                return f"pxrref_{n}", MODULE_VARS[n]
            raise FtransError(f"{self.name}: unknown name {n}")
        if v.dims is not None:
            raise FtransError(f"{self.name}: array {n} used as scalar")
        if v.dummy:
            return f"(*v_{n})", v.ctype
        return f"v_{n}", v.ctype

    @staticmethod
    def promote(a, b):
        return a if CTYPE_RANK[a] >= CTYPE_RANK[b] else b

    def num(self, t):
        m = re.match(r"((\d+\.\d*|\.\d+|\d+)([edED][+-]?\d+)?)(_(\w+))?$", t)
        body, kind = m.group(1), m.group(5)
        is_real = "." in body or re.search(r"[edED]", body)
        if not is_real:
            if kind in ("idp", "num", "8", "lp"):
                return f"((int64_t){body})", "int64_t"
            return body, "int32_t"
        dexp = "d" in body.lower()
        body_c = body.lower().replace("d", "e")
        if body_c.endswith("."):
            body_c += "0"
        if body_c.startswith("."):
            body_c = "0" + body_c
        if kind in ("num", "8") or dexp:
            return f"{body_c}", "double"
        if kind not in (None, "4"):
            raise FtransError(f"literal kind {kind}")
        return f"{body_c}f", "float"

    def idx(self, v, subs, arrname):
        """Column-major linear index of a reference to array v."""
        terms = []
        for d, s in enumerate(subs):
            e, _ = self.ex(s)
            terms.append(f"((int64_t)({e}) - {arrname}_lo{d})")
        acc = terms[-1]
        for d in range(len(terms) - 2, -1, -1):
            acc = f"{terms[d]} + {arrname}_n{d} * ({acc})"
        return acc

    def arr_base(self, n):
        return f"v_{n}"

    def ex(self, e, elem=None):
        """Return (C text, ctype).  ``elem`` names the flat index variable of
        a whole-array statement: bare array names then mean element-wise."""
        k = e[0]
        if k == "num":
            return self.num(e[1])
        if k == "bool":
            return ("1" if e[1] else "0"), "int32_t"
        if k == "paren":
            c, t = self.ex(e[1], elem)
            return f"({c})", t
        if k == "name":
            v = self.lookup(e[1])
            if v is not None and v.dims is not None:
                if elem is None:
                    raise FtransError(f"{self.name}: whole array {e[1]} in scalar context")
                return f"v_{e[1]}[{elem}]", v.ctype
            return self.scalar_ref(e[1])
        if k == "un":
            c, t = self.ex(e[2], elem)
            if e[1] == "!":
                return f"(!({c}))", "int32_t"
            return f"({e[1]}{c})", t
        if k == "bin":
            op = e[1]
            if op == "**":
                base, bt = self.ex(e[2], elem)
                if e[3][0] == "num" and re.match(r"\d+$", e[3][1]):
                    n = int(e[3][1])
                    if n == 2:
                        return f"(({base})*({base}))", bt
                    if n == 3:
                        return f"((({base})*({base}))*({base}))", bt
                ex_, et = self.ex(e[3], elem)
                t = self.promote(bt, et)
                if CTYPE_RANK[t] < 3:
                    raise FtransError("integer power")
                return f"pow({base}, {ex_})", "double"
            a, ta = self.ex(e[2], elem)
            b, tb = self.ex(e[3], elem)
            cop = {".and.": "&&", ".or.": "||", "/=": "!=", ".eq.": "==", ".ne.": "!=",
                   ".lt.": "<", ".gt.": ">", ".le.": "<=", ".ge.": ">="}.get(op, op)
            if cop in ("&&", "||", "==", "!=", "<", ">", "<=", ">="):
                return f"({a} {cop} {b})", "int32_t"
            return f"({a} {cop} {b})", self.promote(ta, tb)
        if k == "ref":
            n, args = e[1], e[2]
            v = self.lookup(n)
            if v is not None and v.dims is not None:
                if any(a[0] == "range" for a in args):
                    raise FtransError(f"{self.name}: section {n} in expression")
                if len(args) != len(v.dims):
                    raise FtransError(f"{self.name}: rank of {n}")
                return f"v_{n}[{self.idx(v, args, 'b_' + n)}]", v.ctype
            return self.intrinsic(n, args, elem)
        raise FtransError(f"expr node {k}")

    def intrinsic(self, n, args, elem):
        cs = [self.ex(a, elem) for a in args]
        if n == "floor":
            return f"((int32_t)floor((double)({cs[0][0]})))", "int32_t"
        if n == "nint":
            return f"((int32_t)lround((double)({cs[0][0]})))", "int32_t"
        if n == "int":
            return f"((int32_t)({cs[0][0]}))", "int32_t"
        if n == "sqrt":
            c, t = cs[0]
            return (f"sqrtf({c})", "float") if t == "float" else (f"sqrt({c})", "double")
        if n == "abs":
            c, t = cs[0]
            if t == "double":
                return f"fabs({c})", t
            if t == "float":
                return f"fabsf({c})", t
            return f"((int64_t)llabs((long long)({c})))", "int64_t"
        if n in ("min", "max"):
            t = cs[0][1]
            for _, tt in cs[1:]:
                t = self.promote(t, tt)
            fn = {"double": "d", "float": "f", "int64_t": "l", "int32_t": "i"}[t]
            acc = cs[0][0]
            for c, _ in cs[1:]:
                acc = f"pxrref_{n}_{fn}({acc}, {c})"
            return acc, t
        if n == "real" or n == "dble":
            return f"((double)({cs[0][0]}))", "double"
        if n == "mod":
            t = self.promote(cs[0][1], cs[1][1])
            if CTYPE_RANK[t] >= 3:
                return f"fmod({cs[0][0]}, {cs[1][0]})", "double"
            return f"(({cs[0][0]}) % ({cs[1][0]}))", t
        raise FtransError(f"{self.name}: unknown function {n}")

    # -- statements --------------------------------------------------------
    def newtmp(self):
        self.tmp += 1
        return f"t{self.tmp}"

    def translate(self):
        out = []
        sig = []
        for a in self.args:
            v = self.vars[a]
            sig.append(f"{v.ctype}* v_{a}" if v.dims is not None else f"{v.ctype}* v_{a}")
        out.append(f"void pxrref_{self.name}({', '.join(sig)}) {{")
        # locals
        for n, v in self.vars.items():
            if v.dummy:
                continue
            if v.param is not None:
                c, _ = self.ex(v.param)
                out.append(f"  const {v.ctype} v_{n} = {c};")
            elif v.dims is None:
                out.append(f"  {v.ctype} v_{n} = 0;")
        # array bound variables (specification expressions at entry)
        for n, v in self.vars.items():
            if v.dims is None:
                continue
            if v.alloc:
                out.append(f"  {v.ctype}* v_{n} = 0;")
                for d in range(len(v.dims)):
                    out.append(f"  int64_t b_{n}_lo{d} = 0, b_{n}_n{d} = 0;")
                out.append(f"  int64_t b_{n}_size = 0;")
                continue
            size = []
            for d, (lo, hi) in enumerate(v.dims):
                lc, _ = self.ex(lo)
                hc, _ = self.ex(hi)
                out.append(f"  const int64_t b_{n}_lo{d} = (int64_t)({lc});")
                out.append(f"  const int64_t b_{n}_n{d} = (int64_t)({hc}) - b_{n}_lo{d} + 1;")
                size.append(f"b_{n}_n{d}")
            out.append(f"  const int64_t b_{n}_size = {' * '.join(size)};")
            if not v.dummy:
                # local arrays start at zero (gfortran -finit-local-zero): a
                # routine that reads an element before setting it (the order-2
                # 2-D Esirkepov reads sx0(+-2)) then has one defined meaning
                out.append(f"  {v.ctype} v_{n}[b_{n}_size > 0 ? b_{n}_size : 1];")
                out.append(f"  memset(v_{n}, 0, sizeof(v_{n}));")
        for n, v in self.vars.items():
            out.append(f"  (void)v_{n};")
        depth = 1
        stack = []
        for ln, s in self.body:
            try:
                depth = self.stmt(s, out, depth, stack)
            except FtransError as e:
                raise FtransError(f"{self.src}:{ln}: {e}  [{s}]")
        if stack:
            raise FtransError(f"{self.name}: unclosed block {stack}")
        out.append("}")
        return "\n".join(out)

    def stmt(self, s, out, depth, stack):
        ind = "  " * depth
        low = s.lower()
        if re.match(r"end\s*subroutine\b", low):
            return depth
        if re.match(r"(end\s*do|enddo)$", low):
            kind = stack.pop()
            assert kind == "do", kind
            depth -= 1
            out.append("  " * depth + "}}")
            return depth
        if re.match(r"(end\s*if|endif)$", low):
            kind = stack.pop()
            assert kind == "if", kind
            depth -= 1
            out.append("  " * depth + "}")
            return depth
        if re.match(r"end\s*select$", low):
            kind = stack.pop()
            assert kind == "select", kind
            depth -= 1
            out.append("  " * depth + "}}")
            return depth
        if low == "return":
            out.append(ind + "return;")
            return depth
        if low == "else":
            out.append("  " * (depth - 1) + "} else {")
            return depth
        m = re.match(r"else\s*if\s*\((.*)\)\s*then$", low)
        if m:
            c, _ = self.ex(parse_expr(m.group(1)))
            out.append("  " * (depth - 1) + f"}} else if ({c}) {{")
            return depth
        m = re.match(r"do\s+(\w+)\s*=\s*(.*)$", low)
        if m:
            var = m.group(1)
            bnds = split_top(m.group(2))
            lo = self.ex(parse_expr(bnds[0]))[0]
            hi = self.ex(parse_expr(bnds[1]))[0]
            st = self.ex(parse_expr(bnds[2]))[0] if len(bnds) > 2 else "1"
            t = self.newtmp()
            vref, _ = self.scalar_ref(var)
            out.append(ind + f"{{ const int64_t {t}_lo = {lo}, {t}_st = {st};")
            out.append(ind + f"  int64_t {t}_trip = ((int64_t)({hi}) - {t}_lo + {t}_st) / {t}_st;")
            out.append(ind + f"  for ({vref} = {t}_lo; {t}_trip > 0; --{t}_trip, {vref} += {t}_st) {{")
            stack.append("do")
            return depth + 1
        if low.startswith("if"):
            m = re.match(r"if\s*\(", low)
            if m:
                # balanced condition
                dep, j = 0, low.index("(")
                for j in range(low.index("("), len(s)):
                    if s[j] == "(":
                        dep += 1
                    elif s[j] == ")":
                        dep -= 1
                        if dep == 0:
                            break
                cond = s[low.index("(") + 1:j]
                rest = s[j + 1:].strip()
                c, _ = self.ex(parse_expr(cond))
                if rest.lower() == "then":
                    out.append(ind + f"if ({c}) {{")
                    stack.append("if")
                    return depth + 1
                out.append(ind + f"if ({c}) {{")
                self.stmt(rest, out, depth + 1, stack)
                out.append(ind + "}")
                return depth
        m = re.match(r"select\s*case\s*\((.*)\)$", low)
        if m:
            c, t = self.ex(parse_expr(m.group(1)))
            tv = self.newtmp()
            out.append(ind + f"{{ const int64_t {tv} = (int64_t)({c}); int {tv}_first = 1; (void){tv}_first;")
            out.append(ind + f"  if (0) {{")
            stack.append("select")
            self._sel = getattr(self, "_sel", []) + [tv]
            return depth + 1
        m = re.match(r"case\s*\((.*)\)$", low)
        if m:
            tv = self._sel[-1]
            conds = []
            for item in split_top(m.group(1)):
                if ":" in item:
                    lo, hi = split_top(item, ":")
                    cc = []
                    if lo:
                        cc.append(f"{tv} >= (int64_t)({self.ex(parse_expr(lo))[0]})")
                    if hi:
                        cc.append(f"{tv} <= (int64_t)({self.ex(parse_expr(hi))[0]})")
                    conds.append("(" + " && ".join(cc) + ")")
                else:
                    conds.append(f"{tv} == (int64_t)({self.ex(parse_expr(item))[0]})")
            out.append("  " * (depth - 1) + f"}} else if ({' || '.join(conds)}) {{")
            return depth
        if re.match(r"case\s+default$", low):
            out.append("  " * (depth - 1) + "} else {")
            return depth
        m = re.match(r"call\s+(\w+)\s*\((.*)\)$", low)
        if m:
            return self.call(m.group(1), m.group(2), out, depth)
        m = re.match(r"allocate\s*\((.*)\)$", low)
        if m:
            for item in split_top(m.group(1)):
                mm = re.match(r"(\w+)\s*\((.*)\)$", item)
                n = mm.group(1)
                v = self.vars[n]
                dims = self._dims(mm.group(2))
                size = []
                for d, (lo, hi) in enumerate(dims):
                    lc, hc = self.ex(lo)[0], self.ex(hi)[0]
                    out.append(ind + f"b_{n}_lo{d} = (int64_t)({lc}); "
                                     f"b_{n}_n{d} = (int64_t)({hc}) - b_{n}_lo{d} + 1;")
                    size.append(f"b_{n}_n{d}")
                out.append(ind + f"b_{n}_size = {' * '.join(size)};")
                out.append(ind + f"v_{n} = ({v.ctype}*)calloc((size_t)b_{n}_size, sizeof({v.ctype}));")
            return depth
        m = re.match(r"deallocate\s*\((.*)\)$", low)
        if m:
            for n in split_top(m.group(1)):
                out.append(ind + f"free(v_{n}); v_{n} = 0;")
            return depth
        # assignment
        lhs, rhs = self._split_assign(s)
        if lhs is None:
            raise FtransError("unhandled statement")
        le = parse_expr(lhs)
        re_ = parse_expr(rhs)
        if le[0] == "name":
            v = self.lookup(le[1])
            if v is not None and v.dims is not None:
                e = self.newtmp()
                rc, _ = self.ex(re_, elem=e)
                out.append(ind + f"for (int64_t {e} = 0; {e} < b_{le[1]}_size; ++{e}) "
                                 f"v_{le[1]}[{e}] = {rc};")
                return depth
        lc, lt = self.ex(le)
        rc, rt = self.ex(re_)
        out.append(ind + f"{lc} = {rc};")
        return depth

    @staticmethod
    def _split_assign(s):
        depth = 0
        for i, c in enumerate(s):
            if c == "(":
                depth += 1
            elif c == ")":
                depth -= 1
            elif c == "=" and depth == 0:
                prev = s[i - 1] if i else ""
                nxt = s[i + 1] if i + 1 < len(s) else ""
                if prev in "<>/=" or nxt == "=":
                    continue
                return s[:i].strip(), s[i + 1:].strip()
        return None, None

    def call(self, name, argstr, out, depth):
        ind = "  " * depth
        callee = self.known.get(name)
        if callee is None:
            raise FtransError(f"call to untranslated routine {name}")
        acts = [P(tokenize(a)).arg() if a else None for a in split_top(argstr)]
        if len(acts) != len(callee.args):
            raise FtransError(f"{name}: {len(acts)} actual args for {len(callee.args)} dummies")
        cargs = []
        for a, dn in zip(acts, callee.args):
            dv = callee.vars[dn]
            if a[0] == "name":
                v = self.lookup(a[1])
                if v is not None and v.dims is not None:
                    cargs.append(f"v_{a[1]}")
                    continue
                if v is not None:
                    cargs.append(f"v_{a[1]}" if v.dummy else f"&v_{a[1]}")
                    continue
            if a[0] == "ref":
                v = self.lookup(a[1])
                if v is not None and v.dims is not None:
                    subs = [x[1] if x[0] == "range" else x for x in a[2]]
                    if any(s is None for s in subs):
                        raise FtransError("open section")
                    cargs.append(f"&v_{a[1]}[{self.idx(v, subs, 'b_' + a[1])}]")
                    continue
            c, t = self.ex(a)
            cargs.append(f"&({dv.ctype}){{{c}}}")
        out.append(ind + f"pxrref_{name}({', '.join(cargs)});")
        return depth


HEADER = r"""/* Generated from the PICSAR Fortran sources by oracle/ftrans.py.
 * Do not edit; regenerate with `make -C oracle ref`. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

double pxrref_clight = 1.0, pxrref_dt = 0.0, pxrref_mu0 = 1.0, pxrref_eps0 = 1.0;
int64_t pxrref_particle_pusher = 0;

void pxrref_set_module(double clight, double dt, int64_t particle_pusher, double mu0,
                       double eps0) {
  pxrref_clight = clight; pxrref_dt = dt; pxrref_particle_pusher = particle_pusher;
  pxrref_mu0 = mu0; pxrref_eps0 = eps0;
}

static inline double pxrref_min_d(double a, double b) { return a < b ? a : b; }
static inline double pxrref_max_d(double a, double b) { return a > b ? a : b; }
static inline float pxrref_min_f(float a, float b) { return a < b ? a : b; }
static inline float pxrref_max_f(float a, float b) { return a > b ? a : b; }
static inline int64_t pxrref_min_l(int64_t a, int64_t b) { return a < b ? a : b; }
static inline int64_t pxrref_max_l(int64_t a, int64_t b) { return a > b ? a : b; }
static inline int32_t pxrref_min_i(int32_t a, int32_t b) { return a < b ? a : b; }
static inline int32_t pxrref_max_i(int32_t a, int32_t b) { return a > b ? a : b; }
"""


def translate_all(srcdir):
    routines = {}
    order = []
    for rel, names in ROUTINES:
        path = os.path.join(srcdir, rel)
        with open(path) as f:
            pass
        for n in names:
            raw = extract_routine(path, n)
            lines = preprocess(raw)
            r = Routine(n, lines, rel, routines)
            routines[n] = r
            order.append(r)
    protos, bodies = [], []
    for r in order:
        text = r.translate()
        protos.append(text.split("{", 1)[0].rstrip() + ";")
        bodies.append(text)
    return HEADER + "\n" + "\n".join(protos) + "\n\n" + "\n\n".join(bodies) + "\n"


def main(argv):
    if len(argv) != 3:
        print(__doc__)
        return 2
    src = translate_all(argv[1])
    os.makedirs(os.path.dirname(os.path.abspath(argv[2])), exist_ok=True)
    with open(argv[2], "w") as f:
        f.write(src)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
