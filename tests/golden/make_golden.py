#!/usr/bin/env python3
"""Generate golden vectors by EXECUTING the reference Fortran source.

No Fortran compiler exists in this image, so this script translates the
subset of Fortran 90 that original/nemolite2d.f90 uses (DO loops, IF/ELSE IF,
CYCLE, SELECT CASE, ALLOCATE, array sections, SIGN/SQRT/SIN/MIN/MAX/REAL/MOD)
into Python, routine by routine, straight from the source text, and runs it.

Semantics kept:
  * every arithmetic operation is one IEEE-754 double operation rounded to
    nearest (Python floats: no contraction, no reassociation);
  * Fortran's parse tree is kept with explicit parentheses (left-to-right
    binary operators, a leading unary minus applies to the whole first term);
  * SIGN(a,b) = |a| with the sign bit of b (gfortran default);
  * SIN/SQRT call the C library, as gfortran's runtime does;
  * default-kind REAL literals go through float32 (all of them are exact here).

The namelist READ is replaced by the case's values; timer calls, OPEN/WRITE
and the gnuplot `output` routine are skipped (fields are snapshotted at each
`irecord` step instead).  Only this script reads the reference source; the
fixtures it writes (tests/golden/*.npz) are plain numbers.

Usage: python tests/golden/make_golden.py --src <reference>/original/nemolite2d.f90 [--out DIR]
(or set NEMOLITE2D_F90 to that path instead of --src)
"""
import argparse
import math
import os
import re
import sys

import numpy as np

# the reference source: --src, else the NEMOLITE2D_F90 environment variable
DEFAULT_SRC = os.environ.get("NEMOLITE2D_F90")
HERE = os.path.dirname(os.path.abspath(__file__))

# Cases: namelist values (jpiglo/jpjglo include the 2 boundary rows, as the
# reference's namelist files do).  Small enough to interpret in seconds.
CASES = {
    "g10x10_ref128phys": dict(jpiglo=12, jpjglo=12, dx=1000.0, dy=1000.0, dep_const=100.0,
                              nit000=1, nitend=40, irecord=10, rdt=20.0, cbfr=0.00015, visc=0.1),
    "g16x9_ref128phys": dict(jpiglo=18, jpjglo=11, dx=1000.0, dy=1000.0, dep_const=100.0,
                             nit000=1, nitend=30, irecord=10, rdt=20.0, cbfr=0.00015, visc=0.1),
    "g9x14_defaultphys": dict(jpiglo=11, jpjglo=16, dx=1000.0, dy=1000.0, dep_const=100.0,
                              nit000=1, nitend=30, irecord=15, rdt=10.0, cbfr=0.001, visc=100.0),
    "g32x32_ref128phys": dict(jpiglo=34, jpjglo=34, dx=1000.0, dy=1000.0, dep_const=100.0,
                              nit000=1, nitend=100, irecord=25, rdt=20.0, cbfr=0.00015, visc=0.1),
    "g128x128_cfg0": dict(jpiglo=130, jpjglo=130, dx=1000.0, dy=1000.0, dep_const=100.0,
                          nit000=1, nitend=12, irecord=6, rdt=20.0, cbfr=0.00015, visc=0.1),
}

INTRINSICS = {"sign", "sqrt", "sin", "min", "max", "real", "mod", "abs", "int", "sum", "any"}
ARGS = {}


# ---------------------------------------------------------------- lexing
def logical_lines(text):
    """Join '&' continuations and strip '!' comments (no strings contain '!'
    in the routines translated here, except format strings we skip)."""
    out, buf = [], ""
    for raw in text.splitlines():
        line = raw
        # strip comment outside of quotes
        q, cut = None, None
        for k, ch in enumerate(line):
            if q:
                if ch == q:
                    q = None
            elif ch in "'\"":
                q = ch
            elif ch == "!":
                cut = k
                break
        if cut is not None:
            line = line[:cut]
        line = line.rstrip()
        s = line.strip()
        if buf:
            if s.startswith("&"):
                s = s[1:]
            buf += " " + s.strip()
        else:
            buf = s
        if buf.endswith("&"):
            buf = buf[:-1]
            continue
        if buf.strip():
            out.extend(x.strip() for x in split_semicolons(buf) if x.strip())
        buf = ""
    return out


def split_semicolons(s):
    parts, q, cur = [], None, ""
    for ch in s:
        if q:
            if ch == q:
                q = None
        elif ch in "'\"":
            q = ch
        elif ch == ";":
            parts.append(cur)
            cur = ""
            continue
        cur += ch
    parts.append(cur)
    return parts


TOKEN_RE = re.compile(r"""
    (?P<num>(\d+\.\d*|\.\d+|\d+)([eEdD][-+]?\d+)?(_\w+)?) |
    (?P<logop>\.(or|and|not|eq|ne|lt|le|gt|ge|true|false)\.) |
    (?P<op>==|/=|<=|>=|\*\*|[-+*/(),:<>=%]) |
    (?P<name>[A-Za-z_]\w*) |
    (?P<str>'[^']*'|"[^"]*") |
    (?P<ws>\s+)
""", re.X | re.I)


def tokenize(s):
    toks, pos = [], 0
    while pos < len(s):
        m = TOKEN_RE.match(s, pos)
        if not m:
            raise SyntaxError("cannot tokenize: %r" % s[pos:])
        pos = m.end()
        kind = m.lastgroup
        if kind == "ws":
            continue
        toks.append((kind, m.group(kind)))
    return toks


def lit(num):
    """Fortran literal -> Python source of the exact double value."""
    m = re.match(r"^([0-9.]+(?:[eEdD][-+]?\d+)?)(_\w+)?$", num)
    body, kind = m.group(1), m.group(2)
    is_real = ("." in body) or re.search(r"[eEdD]", body)
    if not is_real:
        return str(int(body))
    dbl = bool(kind) or "d" in body.lower()
    val = float(body.lower().replace("d", "e"))
    if not dbl:
        val = float(np.float32(val))  # default REAL kind
    return repr(val)


# ---------------------------------------------------------------- parsing
class ExprParser:
    def __init__(self, toks, arrays):
        self.t, self.i, self.arrays = toks, 0, arrays

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else (None, None)

    def take(self, val=None):
        tok = self.peek()
        if val is not None and (tok[1] is None or tok[1].lower() != val):
            raise SyntaxError("expected %r got %r" % (val, tok))
        self.i += 1
        return tok

    def parse(self):
        e = self.or_expr()
        return e

    def or_expr(self):
        e = self.and_expr()
        while self.peek()[1] and self.peek()[1].lower() == ".or.":
            self.take()
            e = "(%s or %s)" % (e, self.and_expr())
        return e

    def and_expr(self):
        e = self.not_expr()
        while self.peek()[1] and self.peek()[1].lower() == ".and.":
            self.take()
            e = "(%s and %s)" % (e, self.not_expr())
        return e

    def not_expr(self):
        if self.peek()[1] and self.peek()[1].lower() == ".not.":
            self.take()
            return "(not %s)" % self.not_expr()
        return self.rel_expr()

    RELOPS = {"==": "==", "/=": "!=", "<": "<", "<=": "<=", ">": ">", ">=": ">=",
              ".eq.": "==", ".ne.": "!=", ".lt.": "<", ".le.": "<=", ".gt.": ">", ".ge.": ">="}

    def rel_expr(self):
        e = self.add_expr()
        op = self.peek()[1]
        if op and op.lower() in self.RELOPS:
            self.take()
            e = "(%s %s %s)" % (e, self.RELOPS[op.lower()], self.add_expr())
        return e

    def add_expr(self):
        # Fortran: [sign] add-operand { add-op add-operand }; a leading sign
        # negates the whole first multiplicative term.
        sign = None
        if self.peek()[1] in ("-", "+"):
            sign = self.take()[1]
        e = self.mult_expr()
        if sign == "-":
            e = "(-%s)" % e
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            e = "(%s %s %s)" % (e, op, self.mult_expr())
        return e

    def mult_expr(self):
        e = self.power()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            e = "(%s %s %s)" % (e, op, self.power())
        return e

    def power(self):
        b = self.primary()
        if self.peek()[1] == "**":
            self.take()
            return "(%s ** %s)" % (b, self.power())
        return b

    def args(self):
        """Parse '(' arg {, arg} ')' where arg may be a section a:b / :."""
        self.take("(")
        out = []
        while True:
            if self.peek()[1] == ")":
                break
            if self.peek()[1] == ":":
                self.take()
                hi = None if self.peek()[1] in (",", ")") else self.or_expr()
                out.append(("sec", None, hi))
            else:
                a = self.or_expr()
                if self.peek()[1] == ":":
                    self.take()
                    hi = None if self.peek()[1] in (",", ")") else self.or_expr()
                    out.append(("sec", a, hi))
                elif self.peek()[1] == "=":  # keyword argument (label=..., STAT=...)
                    self.take()
                    out.append(("kw", a, self.or_expr()))
                else:
                    out.append(("val", a, None))
            if self.peek()[1] == ",":
                self.take()
                continue
            break
        self.take(")")
        return out

    def primary(self):
        kind, val = self.peek()
        if kind == "num":
            self.take()
            return lit(val)
        if kind == "logop" and val.lower() in (".true.", ".false."):
            self.take()
            return "True" if val.lower() == ".true." else "False"
        if val == "(":
            self.take()
            e = self.or_expr()
            self.take(")")
            return "(%s)" % e
        if kind == "name":
            self.take()
            name = val.lower()
            if self.peek()[1] == "(":
                a = self.args()
                if name in INTRINSICS:
                    return self.intrinsic(name, a)
                return "%s[%s]" % (name, ", ".join(subscript(x) for x in a))
            return name
        raise SyntaxError("unexpected token %r" % (self.peek(),))

    def intrinsic(self, name, a):
        v = [x[1] for x in a if x[0] == "val"]
        if name == "sign":
            return "_sign(%s, %s)" % (v[0], v[1])
        if name == "sqrt":
            return "math.sqrt(%s)" % v[0]
        if name == "sin":
            return "math.sin(%s)" % v[0]
        if name == "min":
            return "min(%s)" % ", ".join(v)
        if name == "max":
            return "max(%s)" % ", ".join(v)
        if name == "real":
            return "float(%s)" % v[0]
        if name == "mod":
            return "_mod(%s, %s)" % (v[0], v[1])
        if name == "abs":
            return "abs(%s)" % v[0]
        if name == "int":
            return "int(%s)" % v[0]
        if name == "any":
            return "False"  # ANY(ierr /= 0): host allocation does not fail here
        raise SyntaxError(name)


def subscript(x):
    kind, a, b = x
    if kind == "sec":
        return "_sl(%s, %s)" % (a if a is not None else "None", b if b is not None else "None")
    return a


def expr(s, arrays=None):
    p = ExprParser(tokenize(s), arrays)
    e = p.parse()
    if p.i != len(p.t):
        raise SyntaxError("trailing tokens in %r: %r" % (s, p.t[p.i:]))
    return e


# ---------------------------------------------------------------- runtime
class _sl:
    def __init__(self, lo, hi):
        self.lo, self.hi = lo, hi


class FArr:
    """Fortran array with explicit lower bounds; column-major semantics are
    irrelevant for element access, kept for SUM order in checksums."""

    def __init__(self, bounds, dtype):
        self.lb = [b[0] for b in bounds]
        self.ub = [b[1] for b in bounds]
        self.a = np.zeros([b[1] - b[0] + 1 for b in bounds], dtype=dtype)

    def _idx(self, key):
        if not isinstance(key, tuple):
            key = (key,)
        out = []
        for d, k in enumerate(key):
            if isinstance(k, _sl):
                lo = self.lb[d] if k.lo is None else k.lo
                hi = self.ub[d] if k.hi is None else k.hi
                if lo < self.lb[d] or hi > self.ub[d]:
                    raise IndexError("section out of bounds")
                out.append(slice(lo - self.lb[d], hi - self.lb[d] + 1))
            else:
                if k < self.lb[d] or k > self.ub[d]:
                    raise IndexError("index %d out of bounds [%d,%d]" % (k, self.lb[d], self.ub[d]))
                out.append(k - self.lb[d])
        return tuple(out)

    def __getitem__(self, key):
        r = self.a[self._idx(key)]
        if isinstance(r, np.generic):
            return r.item()
        return r

    def __setitem__(self, key, val):
        self.a[self._idx(key)] = val


def _sign(a, b):
    return math.copysign(abs(a), b)


def _mod(a, b):
    return int(math.fmod(a, b))


# ---------------------------------------------------------------- translation
def split_units(lines):
    """Return {subroutine_name: [lines]} and the program's specification part."""
    units, spec, cur, name = {}, [], None, None
    in_contains = False
    for ln in lines:
        low = ln.lower()
        if low.startswith("contains"):
            in_contains = True
            continue
        m = re.match(r"^subroutine\s+(\w+)\s*(\((.*)\))?", low)
        if m:
            name, cur = m.group(1), []
            ARGS[name] = [x.strip() for x in (m.group(3) or "").split(",") if x.strip()]
            continue
        if re.match(r"^end\s+subroutine", low):
            units[name] = cur
            name, cur = None, None
            continue
        if cur is not None:
            cur.append(ln)
        elif not in_contains:
            spec.append(ln)
    return units, spec


DECL_RE = re.compile(r"^(real|integer|character|logical)\b.*?::\s*(.*)$", re.I)


def declared_names(decl_rest):
    names, depth, cur = [], 0, ""
    for ch in decl_rest:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            names.append(cur)
            cur = ""
        else:
            cur += ch
    names.append(cur)
    out = []
    for n in names:
        n = n.strip()
        if not n:
            continue
        out.append(re.match(r"(\w+)", n).group(1).lower())
    return out


def translate_unit(name, lines, globals_, arrays, int_arrays):
    body, locals_, indent = [], set(), 1
    sel_stack = []
    pad = lambda: "    " * indent

    def emit(s):
        body.append(pad() + s)

    for ln in lines:
        low = ln.lower()
        # strip numeric statement labels (e.g. "901 IF ...")
        m = re.match(r"^(\d+)\s+(.*)$", ln)
        if m:
            ln, low = m.group(2), m.group(2).lower()
        if low.startswith("implicit") or low.startswith("namelist"):
            continue
        dm = DECL_RE.match(ln)
        if dm:
            for n in declared_names(dm.group(2)):
                locals_.add(n)
            continue
        if re.match(r"^call\s+timer_", low) or low.startswith(("open", "rewind", "close", "write")):
            continue
        if low.startswith("read"):
            emit("_read_namelist(); ios = 0")
            continue
        if low.startswith("stop"):
            emit("raise RuntimeError(%r)" % ln)
            continue
        m = re.match(r"^do\s+(\w+)\s*=\s*(.*)$", low)
        if m:
            var = m.group(1)
            parts = [expr(p) for p in split_top(ln[ln.index("=") + 1:])]
            step = parts[2] if len(parts) > 2 else "1"
            emit("for %s in range(%s, (%s) + (1 if (%s) > 0 else -1), %s):" % (var, parts[0], parts[1], step, step))
            indent += 1
            continue
        if re.match(r"^end\s*do$", low):
            indent -= 1
            continue
        m = re.match(r"^select\s+case\s*\((.*)\)$", low)
        if m:
            emit("_sel = %s" % expr(ln[ln.index("(") + 1:ln.rindex(")")]))
            sel_stack.append(0)
            continue
        m = re.match(r"^case\s*\((.*)\)$", low)
        if m:
            if sel_stack[-1]:
                indent -= 1
            emit("%s _sel == (%s):" % ("elif" if sel_stack[-1] else "if", expr(m.group(1))))
            sel_stack[-1] += 1
            indent += 1
            emit("pass")
            continue
        if re.match(r"^case\s+default$", low):
            indent -= 1
            emit("else:")
            indent += 1
            emit("pass")
            continue
        if re.match(r"^end\s+select$", low):
            indent -= 1
            sel_stack.pop()
            continue
        if re.match(r"^else\s*if\s*\(", low):
            indent -= 1
            cond = ln[ln.index("(") : ln.lower().rindex("then")]
            emit("elif %s:" % expr(cond))
            indent += 1
            continue
        if re.match(r"^else$", low):
            indent -= 1
            emit("else:")
            indent += 1
            continue
        if re.match(r"^end\s*if$", low):
            indent -= 1
            continue
        if re.match(r"^if\s*\(", low):
            close = matching_paren(ln, ln.index("("))
            cond = expr(ln[ln.index("(") : close + 1])
            rest = ln[close + 1:].strip()
            if rest.lower() == "then":
                emit("if %s:" % cond)
                indent += 1
            else:
                emit("if %s:" % cond)
                indent += 1
                emit_simple(rest, emit, arrays, int_arrays)
                indent -= 1
            continue
        emit_simple(ln, emit, arrays, int_arrays)
    used_globals = sorted(globals_ - locals_ - set(ARGS.get(name, [])))
    src = ["def %s(%s):" % (name, ", ".join(ARGS.get(name, [])))]
    if used_globals:
        src.append("    global " + ", ".join(used_globals))
    src.extend(body)
    src.append("    return None")
    return "\n".join(src)


def matching_paren(s, i):
    depth = 0
    for k in range(i, len(s)):
        if s[k] == "(":
            depth += 1
        elif s[k] == ")":
            depth -= 1
            if depth == 0:
                return k
    raise SyntaxError(s)


def split_top(s):
    parts, depth, cur = [], 0, ""
    for ch in s:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            parts.append(cur)
            cur = ""
        else:
            cur += ch
    parts.append(cur)
    return [p.strip() for p in parts if p.strip()]


def emit_simple(ln, emit, arrays, int_arrays):
    low = ln.lower().strip()
    if low == "cycle":
        emit("continue")
        return
    if low.startswith("stop"):
        emit("raise RuntimeError(%r)" % ln)
        return
    if re.match(r"^call\s+timer_", low):
        emit("pass")
        return
    m = re.match(r"^call\s+(\w+)\s*(\((.*)\))?$", low)
    if m:
        args = ""
        if m.group(3):
            args = ", ".join(expr(a) for a in split_top(ln[ln.index("(") + 1: ln.rindex(")")]))
        emit("%s(%s)" % (m.group(1), args))
        return
    if low.startswith("allocate"):
        inner = ln[ln.index("(") + 1: ln.rindex(")")]
        for item in split_top(inner):
            if "=" in item and item.lower().startswith("stat"):
                continue
            nm = re.match(r"(\w+)\s*\((.*)\)$", item)
            arr, dims = nm.group(1).lower(), split_top(nm.group(2))
            bounds = []
            for d in dims:
                if ":" in d:
                    lo, hi = d.split(":")
                    bounds.append("(%s, %s)" % (expr(lo), expr(hi)))
                else:
                    bounds.append("(1, %s)" % expr(d))
            dt = "np.int64" if arr in int_arrays else "np.float64"
            emit("%s = FArr([%s], %s)" % (arr, ", ".join(bounds), dt))
        emit("ierr = [0] * 12")
        return
    # assignment
    k = find_assign(ln)
    if k is None:
        raise SyntaxError("unhandled statement: %r" % ln)
    lhs, rhs = ln[:k].strip(), ln[k + 1:].strip()
    r = expr(rhs)
    lm = re.match(r"^(\w+)\s*(\((.*)\))?$", lhs)
    name = lm.group(1).lower()
    if lm.group(2):
        subs = ExprParser(tokenize(lhs[lhs.index("("):]), arrays).args()
        emit("%s[%s] = %s" % (name, ", ".join(subscript(x) for x in subs), r))
    elif name in arrays:
        emit("%s.a[...] = %s" % (name, r))
    else:
        emit("%s = %s" % (name, r))


def find_assign(ln):
    depth = 0
    for k, ch in enumerate(ln):
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        elif ch == "=" and depth == 0:
            prev = ln[k - 1] if k else ""
            nxt = ln[k + 1] if k + 1 < len(ln) else ""
            if prev in "<>/=" or nxt == "=":
                continue
            return k
    return None


def build_program(src_text):
    lines = logical_lines(src_text)
    units, spec = split_units(lines)
    arrays, int_arrays, scalars, params = set(), set(), set(), []
    for ln in spec:
        dm = DECL_RE.match(ln)
        if not dm:
            continue
        head = ln[: ln.index("::")].lower()
        names = declared_names(dm.group(2))
        if "allocatable" in head:
            arrays.update(names)
            if head.startswith("integer"):
                int_arrays.update(names)
        elif "parameter" in head:
            for item in split_top(dm.group(2)):
                n, v = item.split("=", 1)
                params.append((n.strip().lower(), expr(v)))
        else:
            scalars.update(names)
    glob = arrays | scalars | {p[0] for p in params} | {"ios", "ierr"}
    code = ["import math", "import numpy as np"]
    for n, v in params:
        code.append("%s = %s" % (n, v))
    for unit in ("setup", "grid", "allocation", "initialisation", "continuity",
                 "momentum", "bc", "next", "step"):
        code.append(translate_unit(unit, units[unit], glob, arrays, int_arrays))
    return "\n\n".join(code), units


def run_case(pysrc, case):
    ns = {"FArr": FArr, "_sl": _sl, "_sign": _sign, "_mod": _mod, "math": math, "np": np,
          "c_float": "c_float", "c_double": "c_double"}
    snaps = {}

    def _read_namelist():
        for k, v in case.items():
            ns[k] = v

    def output():
        istp = ns["istp"]
        snap = {}
        for f in ("sshn", "un", "vn", "ua", "va", "ssha", "sshn_u", "sshn_v"):
            # Fortran-bounded region, stored (ny, nx) C-order = column-major
            snap[f] = ns[f].a.T.copy()
        snaps[istp] = snap

    ns["_read_namelist"] = _read_namelist
    ns["output"] = output
    exec(compile(pysrc, "<nemolite2d.f90>", "exec"), ns)
    ns["setup"]()
    ns["grid"]()
    ns["initialisation"]()
    ns["istp"] = 0
    output()
    for istp in range(ns["nit000"], ns["nitend"] + 1):
        ns["istp"] = istp
        ns["step"]()
    jpi, jpj = ns["jpi"], ns["jpj"]
    # field_checksum(ua(1:jpiglo,1:jpjglo)) -- SUM in array element order
    def csum(arr):
        s = 0.0
        blk = arr[_sl(1, jpi), _sl(1, jpj)]
        for jj in range(blk.shape[1]):
            for ji in range(blk.shape[0]):
                s = s + abs(float(blk[ji, jj]))
        return s
    checks = {"ua": csum(ns["ua"]), "va": csum(ns["va"]), "sshn": csum(ns["sshn"])}
    extra = {"ht": ns["ht"].a.T.copy(), "hu": ns["hu"].a.T.copy(), "hv": ns["hv"].a.T.copy(),
             "xt": ns["xt"].a.T.copy(), "yt": ns["yt"].a.T.copy()}
    return snaps, checks, extra, jpi, jpj


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", default=DEFAULT_SRC)
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--cases", nargs="*", default=list(CASES))
    ap.add_argument("--dump", action="store_true", help="print the translated program")
    a = ap.parse_args()
    if not a.src:
        ap.error("name the reference's original/nemolite2d.f90 with --src "
                 "(or the NEMOLITE2D_F90 environment variable)")
    with open(a.src) as fh:
        text = fh.read()
    pysrc, _ = build_program(text)
    if a.dump:
        print(pysrc)
        return
    for name in a.cases:
        case = CASES[name]
        snaps, checks, extra, jpi, jpj = run_case(pysrc, case)
        out = {"jpi": jpi, "jpj": jpj, "records": np.array(sorted(snaps)),
               "ua_checksum": checks["ua"], "va_checksum": checks["va"],
               "sshn_checksum": checks["sshn"]}
        for k, v in case.items():
            out["nml_" + k] = v
        for istp, snap in snaps.items():
            for f, arr in snap.items():
                out["s%05d_%s" % (istp, f)] = arr
        out.update({"grid_" + k: v for k, v in extra.items()})
        path = os.path.join(a.out, name + ".npz")
        np.savez_compressed(path, **out)
        print("%s: jpi=%d jpj=%d records=%s ua=%.8E va=%.8E -> %s"
              % (name, jpi, jpj, sorted(snaps), checks["ua"], checks["va"], path))


if __name__ == "__main__":
    sys.exit(main())
