"""Parser for the reference's modelling and kernel-schedule languages.

Model grammar (guide.md "Modeling Language"; compiler/augur/src/Rv/ParseRv.y
:110-221):
    prog  ::= "(" hparam ("," hparam)* ")" "=>" "{" decl+ "}"
    hparam::= id ":" typ
    decl  ::= ("param" | "data") id ["[" ids "]"] "~" expr [comps] ";"
            | "param" id ["[" ids "]"] ":" typ "=" expr [comps] ";"
    comps ::= comp ("," comp)*      comp ::= "for" id "<-" expr "until" expr
    typ   ::= "Int" | "Real" | "Vec" typ | "Mat" typ | "(" typ ")"
    expr  ::= application, indexing, + - * /, literals, identifiers
Schedule grammar (guide.md "Kernel Language"; ParseRv.y:121-146):
    kern ::= base | kern "(*)" kern
    base ::= HMC [xs] [r, r] | NUTS [xs] [r] | RSlice [xs] [r, r]
           | MWG [x] ~ expr [comps] | ConjGibbs [x] | DiscGibbs [x] | ESlice [x]
Defaults for omitted numbers follow compiler/augur/src/Core/KernSyn.hs:64-117.
"""
import re
from dataclasses import dataclass, field
from typing import List, Optional, Tuple

_TOKEN = re.compile(r"\s*(?:(\d+\.\d*(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+|\d+)|([A-Za-z_][A-Za-z_0-9']*)|"
                    r"(=>|<-|\(\*\)|[()\[\]{},;:~=+\-*/]))")


class RvSyntaxError(ValueError):
    pass


def tokenize(src):
    toks, pos = [], 0
    src = src.strip()
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m or m.end() == pos:
            if src[pos:].strip() == "":
                break
            raise RvSyntaxError("unexpected text at %r" % src[pos:pos + 20])
        num, ident, sym = m.groups()
        toks.append(("num", num) if num else ("id", ident) if ident else ("sym", sym))
        pos = m.end()
    return toks


# ---- expressions ---------------------------------------------------------------
@dataclass
class Num:
    value: float
    is_int: bool


@dataclass
class Var:
    name: str


@dataclass
class Call:
    fn: str
    args: list


@dataclass
class Index:
    base: object
    idx: list


@dataclass
class BinOp:
    op: str
    lhs: object
    rhs: object


@dataclass
class Comp:
    var: str
    lo: object
    hi: object


@dataclass
class Decl:
    kind: str                 # "param" | "data"
    name: str
    idxs: List[str]
    dist: Optional[Call]      # for "~" declarations
    typ: Optional[str]        # for deterministic declarations
    expr: Optional[object]    # for deterministic declarations
    comps: List[Comp] = field(default_factory=list)


@dataclass
class Model:
    hparams: List[Tuple[str, str]]
    decls: List[Decl]

    def decl(self, name):
        for d in self.decls:
            if d.name == name:
                return d
        raise KeyError(name)


class _P:
    def __init__(self, toks):
        self.t, self.i = toks, 0

    def peek(self, k=0):
        return self.t[self.i + k] if self.i + k < len(self.t) else ("eof", None)

    def next(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, kind, val=None):
        tok = self.next()
        if tok[0] != kind or (val is not None and tok[1] != val):
            raise RvSyntaxError("expected %s %s, got %s" % (kind, val or "", tok))
        return tok[1]

    def accept(self, kind, val=None):
        tok = self.peek()
        if tok[0] == kind and (val is None or tok[1] == val):
            self.i += 1
            return True
        return False

    # typ ::= Int | Real | Vec typ | Mat typ | ( typ )
    def typ(self):
        if self.accept("sym", "("):
            t = self.typ()
            self.expect("sym", ")")
            return t
        name = self.expect("id")
        if name in ("Vec", "Mat"):
            return "%s %s" % (name, self.typ())
        if name not in ("Int", "Real"):
            raise RvSyntaxError("unknown type %s" % name)
        return name

    def expr(self):
        lhs = self.term()
        while self.peek() in (("sym", "+"), ("sym", "-")):
            op = self.next()[1]
            lhs = BinOp(op, lhs, self.term())
        return lhs

    def term(self):
        lhs = self.factor()
        while self.peek() in (("sym", "*"), ("sym", "/")):
            op = self.next()[1]
            lhs = BinOp(op, lhs, self.factor())
        return lhs

    def factor(self):
        tok = self.next()
        if tok[0] == "num":
            e = Num(float(tok[1]), "." not in tok[1] and "e" not in tok[1].lower())
        elif tok == ("sym", "-"):
            e = BinOp("-", Num(0.0, False), self.factor())
        elif tok == ("sym", "("):
            e = self.expr()
            self.expect("sym", ")")
        elif tok[0] == "id":
            if self.accept("sym", "("):
                args = [] if self.peek() == ("sym", ")") else self.exprs()
                self.expect("sym", ")")
                e = Call(tok[1], args)
            else:
                e = Var(tok[1])
        else:
            raise RvSyntaxError("unexpected %s" % (tok,))
        while self.accept("sym", "["):
            e = Index(e, self.exprs())
            self.expect("sym", "]")
        return e

    def exprs(self):
        out = [self.expr()]
        while self.accept("sym", ","):
            out.append(self.expr())
        return out

    def comps(self):
        out = []
        if self.peek() == ("id", "for"):
            self.expect("id", "for")
            while True:
                self.accept("id", "for")     # "for d <- .., n <- .." or "for .., for .."
                v = self.expect("id")
                self.expect("sym", "<-")
                lo = self.expr()
                self.expect("id", "until")
                hi = self.expr()
                out.append(Comp(v, lo, hi))
                if not self.accept("sym", ","):
                    break
        return out


def parse_model(src):
    p = _P(tokenize(src))
    p.expect("sym", "(")
    hps = []
    while True:
        name = p.expect("id")
        p.expect("sym", ":")
        hps.append((name, p.typ()))
        if not p.accept("sym", ","):
            break
    p.expect("sym", ")")
    p.expect("sym", "=>")
    p.expect("sym", "{")
    decls = []
    while not p.accept("sym", "}"):
        kind = p.expect("id")
        if kind not in ("param", "data"):
            raise RvSyntaxError("declaration must start with param or data, got %s" % kind)
        name = p.expect("id")
        idxs = []
        if p.accept("sym", "["):
            idxs.append(p.expect("id"))
            while p.accept("sym", ","):
                idxs.append(p.expect("id"))
            p.expect("sym", "]")
        if p.accept("sym", "~"):
            dist = p.expr()
            if not isinstance(dist, Call):
                raise RvSyntaxError("%s: expected a distribution after ~" % name)
            d = Decl(kind, name, idxs, dist, None, None)
        else:
            p.expect("sym", ":")
            typ = p.typ()
            p.expect("sym", "=")
            d = Decl(kind, name, idxs, None, typ, p.expr())
        d.comps = p.comps()
        p.expect("sym", ";")
        decls.append(d)
    if p.peek()[0] != "eof":
        raise RvSyntaxError("trailing text after the model")
    return Model(hps, decls)


# ---- schedules --------------------------------------------------------------------
@dataclass
class Kern:
    kind: str                      # HMC NUTS RSlice MWG ConjGibbs DiscGibbs ESlice
    vars: List[str]
    params: List[float]
    proposal: Optional[object] = None
    comps: List[Comp] = field(default_factory=list)


_DEFAULTS = {"HMC": [1.0, 0.05], "RSlice": [1.0, 0.05], "NUTS": [0.05]}   # KernSyn.hs:64-117


def parse_schedule(src):
    out = []
    for part in src.split("(*)"):
        p = _P(tokenize(part))
        kind = p.expect("id")
        if kind not in ("HMC", "NUTS", "RSlice", "MWG", "ConjGibbs", "DiscGibbs", "ESlice"):
            raise RvSyntaxError("unknown kernel %s" % kind)
        p.expect("sym", "[")
        vs = [p.expect("id")]
        while p.accept("sym", ","):
            vs.append(p.expect("id"))
        p.expect("sym", "]")
        k = Kern(kind, vs, list(_DEFAULTS.get(kind, [])))
        if kind in _DEFAULTS and p.accept("sym", "["):
            nums = [p.expr()]
            while p.accept("sym", ","):
                nums.append(p.expr())
            p.expect("sym", "]")
            k.params = [float(_const(n)) for n in nums]
            if len(k.params) != len(_DEFAULTS[kind]):
                raise RvSyntaxError("%s takes %d numbers" % (kind, len(_DEFAULTS[kind])))
        if kind == "MWG":
            p.expect("sym", "~")
            k.proposal = p.expr()
            k.comps = p.comps()
        if p.peek()[0] != "eof":
            raise RvSyntaxError("trailing text in kernel %r" % part.strip())
        out.append(k)
    return out


def _const(e):
    if isinstance(e, Num):
        return e.value
    if isinstance(e, BinOp) and e.op == "-" and isinstance(e.lhs, Num) and e.lhs.value == 0.0:
        return -_const(e.rhs)
    raise RvSyntaxError("expected a number")


def const_value(e, env):
    """Value of a literal or a hyper-parameter name in env."""
    if isinstance(e, Num):
        return e.value
    if isinstance(e, Var) and e.name in env:
        return env[e.name]
    if isinstance(e, BinOp) and e.op == "-" and isinstance(e.lhs, Num) and e.lhs.value == 0.0:
        return -const_value(e.rhs, env)
    raise ValueError("not a constant: %r" % (e,))
