"""An interpreter for the subset of Rust that the reference's AIR source files use.

Fixture generation only (tests/golden/make_air_vectors.py): it parses the
reference's `.rs` files (free functions, constants, structs, inherent `impl`
blocks and `Lazy` statics; trait impls are skipped) and evaluates their
constraint evaluators and layout builders on seeded inputs, so
that the golden vectors come from the reference's own code rather than from a
restatement of it. Nothing at test time imports this module.

Values: Goldilocks field elements are `Fe` (the reference's `F`); Rust integers
are Python ints (casts mask to the target width); vectors, slices and arrays
are Python lists; structs are `Struct` objects; closures and functions are
Python callables. Iterator adaptors are evaluated eagerly over lists.
"""
import re

P = 0xFFFFFFFF00000001
U64 = (1 << 64) - 1


class RustError(Exception):
    pass


# ---------------------------------------------------------------- values
class Fe:
    __slots__ = ("v",)

    def __init__(self, v):
        self.v = v % P

    def _o(self, o):
        if isinstance(o, Fe):
            return o.v
        raise RustError(f"field op with {type(o).__name__}")

    def __add__(self, o):
        return Fe(self.v + self._o(o))

    def __sub__(self, o):
        return Fe(self.v - self._o(o))

    def __mul__(self, o):
        return Fe(self.v * self._o(o))

    def __truediv__(self, o):
        d = self._o(o)
        if d == 0:
            raise RustError("division by zero in F")
        return Fe(self.v * pow(d, P - 2, P))

    def __neg__(self):
        return Fe(-self.v)

    def __eq__(self, o):
        return isinstance(o, Fe) and o.v == self.v

    def __hash__(self):
        return hash(self.v)

    def __repr__(self):
        return f"Fe({self.v})"


class Struct:
    def __init__(self, name, fields):
        self.__dict__["_name"] = name
        self.__dict__["_f"] = dict(fields)

    def __getattr__(self, k):
        try:
            return self.__dict__["_f"][k]
        except KeyError:
            raise AttributeError(k)

    def get(self, k):
        return self._f[k]

    def set(self, k, v):
        self._f[k] = v

    def clone(self):
        return Struct(self._name, {k: _clone(v) for k, v in self._f.items()})


def _clone(v):
    if isinstance(v, list):
        return [_clone(x) for x in v]
    if isinstance(v, Struct):
        return v.clone()
    return v


class RRange:
    def __init__(self, lo, hi, inclusive):
        self.lo, self.hi, self.inclusive = lo, hi, inclusive

    def items(self):
        lo = 0 if self.lo is None else self.lo
        hi = self.hi + 1 if self.inclusive else self.hi
        return list(range(lo, hi))

    def contains(self, x):
        if self.lo is not None and x < self.lo:
            return False
        if self.hi is None:
            return True
        return x <= self.hi if self.inclusive else x < self.hi


class Ref:
    """`&mut x` of a local holding an immutable value (an integer): reads and
    writes go through to the variable."""
    __slots__ = ("scope", "name")

    def __init__(self, scope, name):
        self.scope, self.name = scope, name

    def get(self):
        return self.scope.vars[self.name]

    def set(self, v):
        self.scope.vars[self.name] = v


def dv(v):
    return v.get() if isinstance(v, Ref) else v


class Ret(Exception):
    def __init__(self, v):
        self.v = v


class Brk(Exception):
    def __init__(self, v=None, label=None):
        self.v = v
        self.label = label


class Cont(Exception):
    def __init__(self, label=None):
        self.label = label


# ---------------------------------------------------------------- lexer
_TOK = re.compile(r"""
  (?P<ws>\s+)
 |(?P<lc>//[^\n]*)
 |(?P<str>b?"(?:\\[\s\S]|[^"\\])*")
 |(?P<chr>b?'(?:\\.|[^'\\])')
 |(?P<life>'[A-Za-z_][A-Za-z0-9_]*)
 |(?P<num>0x[0-9A-Fa-f_]+(?:[iu](?:8|16|32|64|128|size))?|0b[01_]+(?:[iu](?:8|16|32|64|128|size))?|[0-9][0-9_]*(?:[iu](?:8|16|32|64|128|size))?)
 |(?P<id>[A-Za-z_][A-Za-z0-9_]*)
 |(?P<op><<=|>>=|\.\.=|\.\.\.|::|->|=>|==|!=|<=|>=|&&|\|\||\+=|-=|\*=|/=|%=|\^=|&=|\|=|<<|>>|\.\.|[-+*/%^!&|<>=.,;:#?@$~(){}\[\]])
""", re.X)


def lex(src):
    out = []
    i, n = 0, len(src)
    while i < n:
        if src.startswith("/*", i):
            depth, j = 0, i
            while j < n:
                if src.startswith("/*", j):
                    depth += 1
                    j += 2
                elif src.startswith("*/", j):
                    depth -= 1
                    j += 2
                    if depth == 0:
                        break
                else:
                    j += 1
            i = j
            continue
        m = _TOK.match(src, i)
        if not m:
            raise RustError(f"lex error at {src[i:i + 40]!r}")
        k = m.lastgroup
        t = m.group(k)
        i = m.end()
        if k in ("ws", "lc"):
            continue
        if k == "num":
            mm = re.match(r"(0x[0-9A-Fa-f_]+|0b[01_]+|[0-9][0-9_]*)", t)
            body = mm.group(1).replace("_", "")
            out.append(("num", int(body, 0)))
        elif k == "str":
            out.append(("str", t))
        elif k == "chr":
            out.append(("chr", t))
        elif k == "life":
            out.append(("life", t))
        elif k == "id":
            out.append(("id", t))
        else:
            out.append(("op", t))
    out.append(("eof", None))
    return out


# ---------------------------------------------------------------- parser
KEYWORDS = {"let", "mut", "fn", "if", "else", "for", "in", "while", "loop", "return", "break", "continue",
            "match", "as", "const", "static", "struct", "pub", "use", "mod", "impl", "enum", "type", "move",
            "ref", "true", "false", "where", "unsafe", "crate", "dyn", "trait"}

BIN_PREC = {"||": 3, "&&": 4, "==": 5, "!=": 5, "<": 5, ">": 5, "<=": 5, ">=": 5, "|": 6, "^": 7, "&": 8,
            "<<": 9, ">>": 9, "+": 10, "-": 10, "*": 11, "/": 11, "%": 11}


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0
        self.macros = {}
        self._impl_type = None

    # -- token helpers
    def peek(self, k=0):
        return self.t[self.i + k]

    def at(self, v, k=0):
        tk = self.t[self.i + k]
        return tk[1] == v and tk[0] in ("op", "id")

    def next(self):
        tk = self.t[self.i]
        self.i += 1
        return tk

    def expect(self, v):
        tk = self.next()
        if tk[1] != v:
            raise RustError(f"expected {v!r}, got {tk!r} near {self.context()}")
        return tk

    def ident(self):
        tk = self.next()
        if tk[0] != "id":
            raise RustError(f"expected identifier, got {tk!r} near {self.context()}")
        return tk[1]

    def context(self):
        return " ".join(str(x[1]) for x in self.t[max(0, self.i - 8):self.i + 8])

    def skip_balanced(self):
        """skip one token tree: a bracketed group or a single token"""
        o = self.next()[1]
        close = {"(": ")", "[": "]", "{": "}"}.get(o)
        if not close:
            return
        depth = 1
        while depth:
            tk = self.next()
            if tk[0] == "eof":
                raise RustError("unbalanced")
            if tk[1] in ("(", "[", "{"):
                depth += 1
            elif tk[1] in (")", "]", "}"):
                depth -= 1

    # -- types: returned as a token list (only array lengths are ever read)
    def parse_type(self, stops):
        start = self.i
        depth = 0
        while True:
            tk = self.peek()
            v = tk[1]
            if tk[0] == "eof":
                break
            if depth == 0 and tk[0] == "op" and v in stops:
                break
            if depth == 0 and tk[0] == "id" and v in stops:
                break
            if v in ("(", "[", "<"):
                depth += 1
            elif v in (")", "]", ">"):
                if depth == 0:
                    break
                depth -= 1
            elif v == ">>":
                if depth == 1:
                    # closes this generic and the enclosing one: split the token
                    self.t[self.i:self.i + 1] = [("op", ">"), ("op", ">")]
                    depth -= 1
                    self.next()
                    continue
                if depth < 2:
                    break
                depth -= 2
            elif v == "->" and depth == 0 and "->" in stops:
                break
            self.next()
        return self.t[start:self.i]

    # -- items
    def parse_items(self, env, until_brace=False):
        while True:
            tk = self.peek()
            if tk[0] == "eof" or (until_brace and tk[1] == "}"):
                return
            self.parse_item(env)

    def skip_attrs(self):
        while self.at("#"):
            self.next()
            if self.at("!"):
                self.next()
            if self.at("["):
                # #[cfg(test)] mod ... { } is skipped by the caller through this flag
                start = self.i
                self.skip_balanced()
                txt = " ".join(str(x[1]) for x in self.t[start:self.i])
                if "cfg ( test )" in txt:
                    self._skip_next_item = True

    def skip_vis(self):
        if self.at("pub"):
            self.next()
            if self.at("("):
                self.skip_balanced()

    def parse_item(self, env):
        self._skip_next_item = False
        self.skip_attrs()
        skip = self._skip_next_item
        self.skip_vis()
        tk = self.peek()
        v = tk[1]
        if v == "use" or v == "extern":
            toks = []
            while not self.at(";"):
                toks.append(self.next())
            self.next()
            for j in range(1, len(toks) - 1):  # `use path::{X as Y}`: Y names X
                if toks[j][1] == "as" and toks[j - 1][0] == "id" and toks[j + 1][0] == "id":
                    env.aliases[toks[j + 1][1]] = toks[j - 1][1]
        elif v == "mod":
            self.next()
            self.ident()
            if self.at(";"):
                self.next()
            else:
                if skip:
                    self.skip_balanced()
                else:
                    self.expect("{")
                    self.parse_items(env, until_brace=True)
                    self.expect("}")
        elif v in ("const", "static") and not (self.peek(1)[1] == "fn"):
            self.next()
            if self.at("mut"):
                self.next()
            name = self.ident()
            self.expect(":")
            ty = self.parse_type({"="})
            self.expect("=")
            e = self.parse_expr()
            self.expect(";")
            if not skip:
                env.consts[name] = (e, ty)
        elif v == "fn" or (v == "const" and self.peek(1)[1] == "fn") or v == "unsafe":
            if v in ("const", "unsafe"):
                self.next()
            self.expect("fn")
            name = self.ident()
            if self.at("<"):
                self.parse_type({"("})
                # parse_type stops at the closing '>' of the generics
                if self.at(">"):
                    self.next()
            self.expect("(")
            params = []
            while not self.at(")"):
                j = 0
                while self.peek(j)[1] in ("&", "mut"):
                    j += 1
                if self.peek(j)[1] == "self" and self.peek(j + 1)[1] in (",", ")"):
                    self.i += j + 1
                    params.append((("pid", "self"), None))
                else:
                    pat = self.parse_pattern()
                    self.expect(":")
                    ty = self.parse_type({",", ")"})
                    params.append((pat, ty))
                if self.at(","):
                    self.next()
            self.expect(")")
            if self.at("->"):
                self.next()
                self.parse_type({"{", "where"})
            if self.at("where"):
                while not self.at("{"):
                    self.next()
            body = self.parse_block()
            if not skip:
                env.fns[name] = ("fn", name, params, body)
        elif v == "struct" or v == "enum" or v == "union":
            self.next()
            name = self.ident()
            if self.at("<"):
                self.parse_type({"{", "(", ";"})
                if self.at(">"):
                    self.next()
            if self.at("where"):
                while not self.at("{"):
                    self.next()
            if self.at(";"):
                self.next()
            elif self.at("("):
                self.skip_balanced()
                if self.at(";"):
                    self.next()
            else:
                self.skip_balanced()
        elif v == "trait":
            self.next()
            while not self.at("{"):
                self.next()
            self.skip_balanced()
        elif v == "impl":
            # inherent impl: its functions are registered as "Type::name"; trait impls are skipped
            self.next()
            if self.at("<"):
                self.next()
                self.parse_type({">"})
                self.expect(">")
            head = []
            while not self.at("{"):
                head.append(self.next())
            if skip or any(t[1] == "for" for t in head):
                self.skip_balanced()
            else:
                tname = head[0][1]
                self.expect("{")
                sub = Module()
                old = self._impl_type
                self._impl_type = tname
                try:
                    self.parse_items(sub, until_brace=True)
                finally:
                    self._impl_type = old
                self.expect("}")
                for fname, f in sub.fns.items():
                    env.fns[f"{tname}::{fname}"] = f[:4] + (tname,)
                for cname, c in sub.consts.items():
                    env.consts[f"{tname}::{cname}"] = c
        elif v == "type":
            while not self.at(";"):
                self.skip_balanced()
            self.next()
        elif v == "macro_rules":
            self.next()
            self.expect("!")
            self.ident()
            self.skip_balanced()
        elif v == ";":
            self.next()
        else:
            raise RustError(f"unexpected item token {tk!r} near {self.context()}")

    # -- patterns
    def parse_pattern(self):
        first = self.parse_pattern1()
        if self.at("|") and not getattr(self, "_closure_params", False):
            alts = [first]
            while self.at("|"):
                self.next()
                alts.append(self.parse_pattern1())
            return ("por", alts)
        return first

    def parse_pattern1(self):
        tk = self.peek()
        v = tk[1]
        if v == "&":
            self.next()
            if self.at("mut"):
                self.next()
            return self.parse_pattern1()
        if v == "mut" or v == "ref":
            self.next()
            if self.at("mut"):
                self.next()
            return self.parse_pattern1()
        if v == "(":
            self.next()
            ps = []
            while not self.at(")"):
                ps.append(self.parse_pattern())
                if self.at(","):
                    self.next()
            self.next()
            return ("ptuple", ps)
        if v == "[":
            self.next()
            ps = []
            while not self.at("]"):
                ps.append(self.parse_pattern())
                if self.at(","):
                    self.next()
            self.next()
            return ("ptuple", ps)
        if v == "_" and tk[0] == "id":
            self.next()
            return ("pwild",)
        if tk[0] in ("num", "str", "chr") or v in ("true", "false") or v == "-":
            e = self.parse_unary()
            if self.at("..=") or self.at(".."):
                inc = self.next()[1] == "..="
                hi = self.parse_unary()
                return ("prange", e, hi, inc)
            return ("plit", e)
        if tk[0] == "id":
            path = [self.ident()]
            while self.at("::"):
                self.next()
                path.append(self.ident())
            if self.at("("):
                self.next()
                ps = []
                while not self.at(")"):
                    ps.append(self.parse_pattern())
                    if self.at(","):
                        self.next()
                self.next()
                return ("penum", path, ps)
            if self.at("{"):
                self.skip_balanced()
                return ("penum", path, None)
            if len(path) == 1 and (path[0][0].islower() or path[0] == "_"):
                if self.at("@"):
                    self.next()
                    return ("pbind", path[0], self.parse_pattern1())
                return ("pid", path[0])
            return ("ppath", path)
        raise RustError(f"bad pattern near {self.context()}")

    # -- blocks and statements
    def parse_block(self):
        self.expect("{")
        stmts = []
        tail = None
        while not self.at("}"):
            s, is_tail = self.parse_stmt()
            if s is None:
                continue
            if is_tail:
                tail = s
                if not self.at("}"):
                    raise RustError(f"expression without ';' before {self.context()}")
            else:
                stmts.append(s)
        self.expect("}")
        return ("block", stmts, tail)

    def parse_stmt(self):
        self._skip_next_item = False
        self.skip_attrs()
        if self._skip_next_item:
            # #[cfg(test)] on a statement: skip it
            self.parse_stmt()
            return None, False
        if self.at(";"):
            self.next()
            return None, False
        if self.at("let"):
            self.next()
            pat = self.parse_pattern()
            ty = None
            if self.at(":"):
                self.next()
                ty = self.parse_type({"=", ";"})
            e = None
            if self.at("="):
                self.next()
                e = self.parse_expr()
            if self.at("else"):
                self.next()
                els = self.parse_block()
                self.expect(";")
                return ("letelse", pat, e, els), False
            self.expect(";")
            return ("let", pat, ty, e), False
        if self.at("fn") or (self.at("const") and self.peek(1)[0] == "id") or self.at("use") or self.at("struct"):
            self.parse_item(self.local_items)
            return None, False
        if self.at("macro_rules") and self.at("!", 1):
            self.next()
            self.next()
            self.parse_macro_rules()
            return None, False
        if self.peek()[0] == "life" and self.at(":", 1):
            e = self.parse_primary()
            if self.at(";"):
                self.next()
            return ("expr", e), False
        if self.peek()[1] in ("if", "for", "while", "loop", "match", "unsafe", "{") and self.peek()[0] in ("id", "op"):
            # a block-like expression in statement position ends at its closing brace
            e = self.parse_primary()
            if self.at(";"):
                self.next()
                return ("expr", e), False
            if self.at("}"):
                return e, True
            if self.at(".") or self.at("?"):
                e = self.parse_postfix(e)
                if self.at(";"):
                    self.next()
                    return ("expr", e), False
                return e, True
            return ("expr", e), False
        e = self.parse_expr(stmt=True)
        if self.at(";"):
            self.next()
            return ("expr", e), False
        if self.at("}"):
            return e, True
        if e[0] in ("if", "for", "while", "loop", "block", "match", "unsafe"):
            return ("expr", e), False
        raise RustError(f"missing ';' near {self.context()}")

    # -- expressions
    def parse_expr(self, stmt=False, no_struct=False):
        old = getattr(self, "_no_struct", False)
        self._no_struct = no_struct
        try:
            return self.parse_assign(stmt)
        finally:
            self._no_struct = old

    def parse_assign(self, stmt):
        lhs = self.parse_range()
        tk = self.peek()
        if tk[0] == "op" and tk[1] in ("=", "+=", "-=", "*=", "/=", "%=", "^=", "&=", "|=", "<<=", ">>="):
            self.next()
            rhs = self.parse_assign(False)
            return ("assign", tk[1], lhs, rhs)
        return lhs

    def parse_range(self):
        if self.at("..") or self.at("..="):
            inc = self.next()[1] == "..="
            if self._range_end():
                return ("range", None, None, inc)
            return ("range", None, self.parse_bin(3), inc)
        lo = self.parse_bin(3)
        if self.at("..") or self.at("..="):
            inc = self.next()[1] == "..="
            if self._range_end():
                return ("range", lo, None, inc)
            return ("range", lo, self.parse_bin(3), inc)
        return lo

    def _range_end(self):
        tk = self.peek()
        return tk[1] in (")", "]", "}", ",", ";", "=>") or (tk[1] == "{" and self._no_struct)

    def parse_bin(self, minp):
        lhs = self.parse_unary()
        while True:
            tk = self.peek()
            if tk[0] == "id" and tk[1] == "as":
                self.next()
                ty = self.parse_type({",", ")", ";", "]", "}", "+", "-", "*", "/", "%", "<<", ">>", "&", "|", "^",
                                      "==", "!=", "<", ">", "<=", ">=", "&&", "||", "..", "..=", "{", "as", "=>"})
                lhs = ("cast", lhs, " ".join(str(x[1]) for x in ty))
                continue
            if tk[0] != "op" or tk[1] not in BIN_PREC:
                return lhs
            p = BIN_PREC[tk[1]]
            if p < minp:
                return lhs
            self.next()
            rhs = self.parse_bin(p + 1)
            lhs = ("bin", tk[1], lhs, rhs)

    def parse_unary(self):
        tk = self.peek()
        if tk[0] == "op" and tk[1] in ("-", "!", "*"):
            self.next()
            return ("un", tk[1], self.parse_unary())
        if tk[0] == "op" and tk[1] in ("&", "&&"):
            self.next()
            if self.at("mut"):
                self.next()
                return ("refmut", self.parse_unary())
            return self.parse_unary()
        return self.parse_postfix(self.parse_primary())

    def parse_args(self, close=")"):
        args = []
        while not self.at(close):
            args.append(self.parse_expr())
            if self.at(","):
                self.next()
        self.expect(close)
        return args

    def parse_postfix(self, e):
        while True:
            if self.at("("):
                self.next()
                e = ("call", e, self.parse_args())
            elif self.at("["):
                self.next()
                idx = self.parse_expr()
                self.expect("]")
                e = ("index", e, idx)
            elif self.at("?"):
                self.next()
                e = ("try", e)
            elif self.at("."):
                self.next()
                tk = self.next()
                if tk[0] == "num":
                    e = ("tindex", e, tk[1])
                    continue
                name = tk[1]
                if self.at("::"):
                    self.next()
                    self.expect("<")
                    self.parse_type({">"})
                    self.expect(">")
                if self.at("("):
                    self.next()
                    e = ("mcall", e, name, self.parse_args())
                else:
                    e = ("field", e, name)
            else:
                return e

    def parse_closure(self):
        if self.at("move"):
            self.next()
        params = []
        if self.at("||"):
            self.next()
        else:
            self.expect("|")
            self._closure_params = True
            try:
                while not self.at("|"):
                    pat = self.parse_pattern()
                    if self.at(":"):
                        self.next()
                        self.parse_type({",", "|"})
                    params.append(pat)
                    if self.at(","):
                        self.next()
            finally:
                self._closure_params = False
            self.expect("|")
        if self.at("->"):
            self.next()
            self.parse_type({"{"})
            body = self.parse_block()
        else:
            body = self.parse_expr()
        return ("closure", params, body)

    def parse_primary(self):
        tk = self.peek()
        k, v = tk
        if k == "life" and self.at(":", 1):
            label = v
            self.next()
            self.next()
            e = self.parse_primary()
            if e[0] not in ("for", "while", "loop"):
                raise RustError(f"label on {e[0]}")
            return ("label", label, e)
        if k == "num":
            self.next()
            return ("lit", v)
        if k == "str":
            self.next()
            return ("lit", v)
        if k == "chr":
            self.next()
            return ("lit", v)
        if v == "(" and k == "op":
            self.next()
            if self.at(")"):
                self.next()
                return ("tuple", [])
            e = self.parse_expr()
            if self.at(","):
                items = [e]
                while self.at(","):
                    self.next()
                    if self.at(")"):
                        break
                    items.append(self.parse_expr())
                self.expect(")")
                return ("tuple", items)
            self.expect(")")
            return e
        if v == "[" and k == "op":
            self.next()
            if self.at("]"):
                self.next()
                return ("array", [])
            first = self.parse_expr()
            if self.at(";"):
                self.next()
                n = self.parse_expr()
                self.expect("]")
                return ("repeat", first, n)
            items = [first]
            while self.at(","):
                self.next()
                if self.at("]"):
                    break
                items.append(self.parse_expr())
            self.expect("]")
            return ("array", items)
        if v == "{" and k == "op":
            return self.parse_block()
        if v in ("|", "||") and k == "op" or v == "move":
            return self.parse_closure()
        if k == "id":
            if v == "if":
                return self.parse_if()
            if v == "match":
                self.next()
                scrut = self.parse_expr(no_struct=True)
                self.expect("{")
                arms = []
                while not self.at("}"):
                    pat = self.parse_pattern()
                    guard = None
                    if self.at("if"):
                        self.next()
                        guard = self.parse_expr()
                    self.expect("=>")
                    body = self.parse_expr()
                    if self.at(","):
                        self.next()
                    arms.append((pat, guard, body))
                self.expect("}")
                return ("match", scrut, arms)
            if v == "for":
                self.next()
                pat = self.parse_pattern()
                self.expect("in")
                it = self.parse_expr(no_struct=True)
                body = self.parse_block()
                return ("for", pat, it, body)
            if v == "while":
                self.next()
                if self.at("let"):
                    raise RustError("while let is not supported")
                cond = self.parse_expr(no_struct=True)
                body = self.parse_block()
                return ("while", cond, body)
            if v == "loop":
                self.next()
                return ("loop", self.parse_block())
            if v == "unsafe":
                self.next()
                return self.parse_block()
            if v == "return":
                self.next()
                if self.at(";") or self.at("}"):
                    return ("return", None)
                return ("return", self.parse_expr())
            if v == "break":
                self.next()
                label = self.next()[1] if self.peek()[0] == "life" else None
                if self.at(";") or self.at("}"):
                    return ("break", None, label)
                return ("break", self.parse_expr(), label)
            if v == "continue":
                self.next()
                label = self.next()[1] if self.peek()[0] == "life" else None
                return ("continue", label)
            if v in ("true", "false"):
                self.next()
                return ("lit", v == "true")
            # path
            path = [self.ident()]
            while self.at("::"):
                self.next()
                if self.at("<"):
                    self.next()
                    self.parse_type({">"})
                    self.expect(">")
                    continue
                path.append(self.ident())
            if self.at("!") and not self.at("=", 1):
                self.next()
                return self.parse_macro(path[-1])
            if self.at("{") and not self._no_struct and path[-1][:1].isupper():
                return self.parse_struct_lit(path)
            return ("path", path)
        raise RustError(f"bad expression at {tk!r} near {self.context()}")

    def parse_if(self):
        self.expect("if")
        if self.at("let"):
            self.next()
            pat = self.parse_pattern()
            self.expect("=")
            scrut = self.parse_expr(no_struct=True)
            then = self.parse_block()
            els = None
            if self.at("else"):
                self.next()
                els = self.parse_if() if self.at("if") else self.parse_block()
            return ("iflet", pat, scrut, then, els)
        cond = self.parse_expr(no_struct=True)
        then = self.parse_block()
        els = None
        if self.at("else"):
            self.next()
            els = self.parse_if() if self.at("if") else self.parse_block()
        return ("if", cond, then, els)

    def parse_struct_lit(self, path):
        self.expect("{")
        fields = []
        base = None
        while not self.at("}"):
            if self.at(".."):
                self.next()
                base = self.parse_expr()
                continue
            name = self.ident()
            if self.at(":"):
                self.next()
                fields.append((name, self.parse_expr()))
            else:
                fields.append((name, ("path", [name])))
            if self.at(","):
                self.next()
        self.expect("}")
        return ("struct", path[-1], fields, base)

    def parse_macro_rules(self):
        """macro_rules! name { ($a:expr, ...) => { body }; ... } -> registered, first rule only"""
        name = self.ident()
        self.expect("{")
        self.expect("(")
        params = []
        while not self.at(")"):
            self.expect("$")
            params.append(self.ident())
            self.expect(":")
            self.ident()
            if self.at(","):
                self.next()
        self.expect(")")
        self.expect("=>")
        start = self.i
        self.skip_balanced()
        body = self.t[start + 1:self.i - 1]
        while not self.at("}"):
            self.skip_balanced()
        self.expect("}")
        self.macros[name] = (params, body)

    def expand_macro(self, name):
        params, body = self.macros[name]
        self.expect("(")
        args, cur, depth = [], [], 0
        while True:
            tk = self.next()
            if tk[1] in ("(", "[", "{"):
                depth += 1
            elif tk[1] in (")", "]", "}"):
                if depth == 0:
                    break
                depth -= 1
            if tk[1] == "," and depth == 0:
                args.append(cur)
                cur = []
            else:
                cur.append(tk)
        if cur:
            args.append(cur)
        if len(args) != len(params):
            raise RustError(f"macro {name}: {len(args)} args")
        sub = dict(zip(params, args))
        out, j = [], 0
        while j < len(body):
            if body[j][1] == "$" and j + 1 < len(body) and body[j + 1][1] in sub:
                out += [("op", "(")] + sub[body[j + 1][1]] + [("op", ")")]
                j += 2
            else:
                out.append(body[j])
                j += 1
        p = Parser(out + [("eof", None)])
        p.local_items = self.local_items
        p.macros = self.macros
        return p.parse_expr()

    def parse_macro(self, name):
        if name == "macro_rules":
            self.parse_macro_rules()
            return ("tuple", [])
        if name in self.macros:
            return self.expand_macro(name)
        open_ = self.peek()[1]
        close = {"(": ")", "[": "]", "{": "}"}[open_]
        if name == "vec":
            self.next()
            if self.at(close):
                self.next()
                return ("array", [])
            first = self.parse_expr()
            if self.at(";"):
                self.next()
                n = self.parse_expr()
                self.expect(close)
                return ("repeat", first, n)
            items = [first]
            while self.at(","):
                self.next()
                if self.at(close):
                    break
                items.append(self.parse_expr())
            self.expect(close)
            return ("array", items)
        if name in ("assert", "assert_eq", "assert_ne", "debug_assert", "debug_assert_eq", "debug_assert_ne",
                    "println", "eprintln", "print", "eprint", "trace", "debug", "info", "warn"):
            self.skip_balanced()
            return ("tuple", [])
        if name in ("panic", "unreachable", "unimplemented", "todo"):
            self.skip_balanced()
            return ("panic", name)
        if name == "format":
            self.skip_balanced()
            return ("lit", "")
        raise RustError(f"unsupported macro {name}!")


class Module:
    """Parsed items of one or more source files."""

    def __init__(self):
        self.fns = {}
        self.consts = {}
        self.aliases = {}
        self.local_items = self


def parse_sources(texts):
    mod = Module()
    for src in texts:
        p = Parser(lex(src))
        p.local_items = mod
        p.parse_items(mod)
    return mod


# ---------------------------------------------------------------- evaluator
_INT_BITS = {"u8": 8, "u16": 16, "u32": 32, "u64": 64, "u128": 128, "usize": 64,
             "i8": -8, "i16": -16, "i32": -32, "i64": -64, "i128": -128, "isize": -64}


def _cast(v, ty):
    ty = ty.strip()
    if ty in _INT_BITS:
        if isinstance(v, bool):
            v = int(v)
        if isinstance(v, Fe):
            raise RustError("cast of a field element")
        b = _INT_BITS[ty]
        if b > 0:
            return v & ((1 << b) - 1)
        b = -b
        v &= (1 << b) - 1
        return v - (1 << b) if v >> (b - 1) else v
    if ty == "F":
        return Fe(v) if not isinstance(v, Fe) else v
    return v


class Scope:
    __slots__ = ("vars", "parent")

    def __init__(self, parent=None):
        self.vars = {}
        self.parent = parent

    def lookup(self, name):
        s = self
        while s is not None:
            if name in s.vars:
                return s
            s = s.parent
        return None


class Interp:
    def __init__(self, mod, extra_builtins=None):
        self.mod = mod
        self.const_cache = {}
        self.builtins = dict(extra_builtins or {})
        self.steps = 0

    # -- entry
    def call(self, name, *args):
        return self.call_fn(self.mod.fns[name], list(args))

    def const(self, name):
        if name in self.const_cache:
            return self.const_cache[name]
        e, ty = self.mod.consts[name]
        v = self.eval(e, Scope())
        self.const_cache[name] = v
        return v

    def call_fn(self, f, args):
        _, name, params, body = f[:4]
        if len(params) != len(args):
            raise RustError(f"{name}: {len(args)} args for {len(params)} params")
        sc = Scope()
        if len(f) > 4:
            sc.vars["Self"] = ("type", f[4])
        for (pat, ty), a in zip(params, args):
            self.bind(pat, a, sc)
        try:
            return self.eval(body, sc)
        except Ret as r:
            return r.v

    # -- patterns
    def bind(self, pat, v, sc):
        k = pat[0]
        if k == "pid":
            sc.vars[pat[1]] = v
        elif k == "pwild":
            pass
        elif k == "ptuple":
            vs = list(v)
            if len(vs) != len(pat[1]):
                raise RustError("tuple pattern arity")
            for p, x in zip(pat[1], vs):
                self.bind(p, x, sc)
        elif k == "pbind":
            sc.vars[pat[1]] = v
            self.bind(pat[2], v, sc)
        elif k == "ppath" and len(pat[1]) == 1:
            sc.vars[pat[1][0]] = v
        else:
            raise RustError(f"irrefutable pattern {k} not supported")

    def matches(self, pat, v, sc):
        k = pat[0]
        if k in ("pwild",):
            return True
        if k == "pid":
            sc.vars[pat[1]] = v
            return True
        if k == "plit":
            return self.eval(pat[1], sc) == v
        if k == "prange":
            lo, hi = self.eval(pat[1], sc), self.eval(pat[2], sc)
            return lo <= v <= hi if pat[3] else lo <= v < hi
        if k == "por":
            return any(self.matches(p, v, sc) for p in pat[1])
        if k == "ptuple":
            vs = list(v)
            return len(vs) == len(pat[1]) and all(self.matches(p, x, sc) for p, x in zip(pat[1], vs))
        if k == "penum":
            name = pat[1][-1]
            if name == "Some":
                if v is None:
                    return False
                return self.matches(pat[2][0], v, sc)
            if name in ("Ok",):
                return self.matches(pat[2][0], v, sc)
            raise RustError(f"enum pattern {name}")
        if k == "ppath":
            name = pat[1][-1]
            if name == "None":
                return v is None
            return v == ("enum", name)
        if k == "pbind":
            if self.matches(pat[2], v, sc):
                sc.vars[pat[1]] = v
                return True
            return False
        raise RustError(f"pattern {k}")

    # -- expressions
    def eval(self, e, sc):
        return getattr(self, "e_" + e[0])(e, sc)

    def e_block(self, e, sc):
        inner = Scope(sc)
        for s in e[1]:
            self.exec_stmt(s, inner)
        return self.eval(e[2], inner) if e[2] is not None else ()

    def exec_stmt(self, s, sc):
        k = s[0]
        if k == "let":
            _, pat, ty, ex = s
            if ex is None:
                self.bind(pat, None, sc)
                return
            if ex[0] == "call" and ex[1][0] == "path" and ex[1][1][-1] == "from_fn" and ty:
                n = self._array_len(ty, sc)
                f = self.eval(ex[2][0], sc)
                self.bind(pat, [f(i) for i in range(n)], sc)
                return
            v = self.eval(ex, sc)
            if ty and len(ty) == 1 and ty[0][1] in _INT_BITS and isinstance(v, int) and not isinstance(v, bool):
                v = _cast(v, ty[0][1])
            self.bind(pat, v, sc)
        elif k == "letelse":
            _, pat, ex, els = s
            v = self.eval(ex, sc)
            tmp = Scope(sc)
            if self.matches(pat, v, tmp):
                sc.vars.update(tmp.vars)
            else:
                self.eval(els, sc)
                raise RustError("let-else fell through")
        elif k == "expr":
            self.eval(s[1], sc)
        else:
            raise RustError(f"stmt {k}")

    def _array_len(self, ty, sc):
        # [T; N]
        toks = ty
        if toks[0][1] != "[":
            raise RustError("from_fn needs an array type")
        j = max(i for i, t in enumerate(toks) if t[1] == ";")
        sub = Parser(list(toks[j + 1:-1]) + [("eof", None)])
        sub.local_items = self.mod
        return self.eval(sub.parse_expr(), sc)

    def e_lit(self, e, sc):
        return e[1]

    def e_tuple(self, e, sc):
        vs = [self.eval(x, sc) for x in e[1]]
        return tuple(vs) if vs else ()

    def e_array(self, e, sc):
        return [self.eval(x, sc) for x in e[1]]

    def e_repeat(self, e, sc):
        v = self.eval(e[1], sc)
        n = self.eval(e[2], sc)
        return [_clone(v) for _ in range(n)]

    def e_panic(self, e, sc):
        raise RustError(f"{e[1]}! reached")

    def e_path(self, e, sc):
        path = e[1]
        name = path[-1]
        if len(path) == 1:
            s = sc.lookup(name)
            if s is not None:
                return s.vars[name]
        name = self.mod.aliases.get(name, name)
        if name in self.mod.consts:
            return self.const(name)
        if name in self.mod.fns:
            f = self.mod.fns[name]
            return lambda *a, f=f: self.call_fn(f, list(a))
        key = "::".join(path[-2:]) if len(path) >= 2 else name
        for cand in (key, name):
            if cand in self.builtins:
                return self.builtins[cand]
        b = BUILTIN_PATHS.get(key) or BUILTIN_PATHS.get(name)
        if b is not None:
            return b
        if name == "None":
            return None
        raise RustError(f"unknown name {'::'.join(path)}")

    def _self_type(self, name, sc):
        if name == "Self":
            s2 = sc.lookup("Self")
            if s2 is None:
                raise RustError("Self outside an impl")
            return s2.vars["Self"][1]
        return name

    def e_struct(self, e, sc):
        _, name, fields, base = e
        name = self._self_type(name, sc)
        d = {}
        if base is not None:
            b = self.eval(base, sc)
            d.update(b._f)
        for k, x in fields:
            d[k] = self.eval(x, sc)
        return Struct(name, d)

    def e_field(self, e, sc):
        v = self.eval(e[1], sc)
        if isinstance(v, Struct):
            return v.get(e[2])
        raise RustError(f"field {e[2]} of {type(v).__name__}")

    def e_tindex(self, e, sc):
        return self.eval(e[1], sc)[e[2]]

    def e_index(self, e, sc):
        v = self.eval(e[1], sc)
        i = self.eval(e[2], sc)
        if isinstance(i, RRange):
            lo = 0 if i.lo is None else i.lo
            hi = len(v) if i.hi is None else (i.hi + 1 if i.inclusive else i.hi)
            if hi > len(v) or lo > hi:
                raise RustError("slice out of range")
            return v[lo:hi]
        if i < 0 or i >= len(v):
            raise RustError(f"index {i} out of range {len(v)}")
        return v[i]

    def e_range(self, e, sc):
        lo = self.eval(e[1], sc) if e[1] is not None else None
        hi = self.eval(e[2], sc) if e[2] is not None else None
        return RRange(lo, hi, e[3])

    def e_cast(self, e, sc):
        return _cast(self.eval(e[1], sc), e[2])

    def e_refmut(self, e, sc):
        x = e[1]
        if x[0] == "path" and len(x[1]) == 1:
            s2 = sc.lookup(x[1][0])
            if s2 is not None:
                val = s2.vars[x[1][0]]
                if isinstance(val, Ref):
                    return val
                if val is None or isinstance(val, (int, bool, Fe)):
                    return Ref(s2, x[1][0])
        return self.eval(x, sc)

    def e_un(self, e, sc):
        v = dv(self.eval(e[2], sc))
        op = e[1]
        if op == "-":
            return -v
        if op == "!":
            if isinstance(v, bool):
                return not v
            return ~v & U64
        return _clone(v)  # deref: `let mut x = *fe;` copies (arrays and Copy structs)

    def e_bin(self, e, sc):
        op = e[1]
        if op == "&&":
            return bool(self.eval(e[2], sc)) and bool(self.eval(e[3], sc))
        if op == "||":
            return bool(self.eval(e[2], sc)) or bool(self.eval(e[3], sc))
        a = dv(self.eval(e[2], sc))
        b = dv(self.eval(e[3], sc))
        return binop(op, a, b)

    def e_assign(self, e, sc):
        _, op, lhs, rhs = e
        v = self.eval(rhs, sc)
        v = dv(v)
        if op != "=":
            cur = dv(self.eval(lhs, sc))
            v = binop(op[:-1], cur, v)
        self.store(lhs, v, sc)
        return ()

    def store(self, lhs, v, sc):
        k = lhs[0]
        if k == "path" and len(lhs[1]) == 1:
            s = sc.lookup(lhs[1][0])
            if s is None:
                raise RustError(f"assignment to unknown {lhs[1][0]}")
            s.vars[lhs[1][0]] = v
        elif k == "index":
            arr = self.eval(lhs[1], sc)
            i = self.eval(lhs[2], sc)
            arr[i] = v
        elif k == "field":
            obj = self.eval(lhs[1], sc)
            obj.set(lhs[2], v)
        elif k == "un":
            inner = lhs[2]
            if inner[0] == "path" and len(inner[1]) == 1:
                s2 = sc.lookup(inner[1][0])
                if s2 is not None and isinstance(s2.vars[inner[1][0]], Ref):
                    s2.vars[inner[1][0]].set(v)
                    return
            self.store(inner, v, sc)
        elif k == "tindex":
            raise RustError("tuple element assignment")
        else:
            raise RustError(f"store to {k}")

    def e_if(self, e, sc):
        if self.eval(e[1], sc):
            return self.eval(e[2], sc)
        if e[3] is not None:
            return self.eval(e[3], sc)
        return ()

    def e_iflet(self, e, sc):
        _, pat, scrut, then, els = e
        v = self.eval(scrut, sc)
        inner = Scope(sc)
        if self.matches(pat, v, inner):
            return self.eval(then, inner)
        if els is not None:
            return self.eval(els, sc)
        return ()

    def e_match(self, e, sc):
        v = self.eval(e[1], sc)
        for pat, guard, body in e[2]:
            inner = Scope(sc)
            if self.matches(pat, v, inner) and (guard is None or self.eval(guard, inner)):
                return self.eval(body, inner)
        raise RustError("no match arm")

    def _iter(self, v):
        if isinstance(v, RRange):
            return v.items()
        if isinstance(v, (list, tuple)):
            return list(v)
        raise RustError(f"cannot iterate {type(v).__name__}")

    def e_label(self, e, sc):
        inner = e[2]
        return getattr(self, "e_" + inner[0])(inner, sc, e[1])

    def e_for(self, e, sc, label=None):
        _, pat, it, body = e
        for x in self._iter(self.eval(it, sc)):
            inner = Scope(sc)
            self.bind(pat, x, inner)
            try:
                self.eval(body, inner)
            except Cont as c:
                if c.label is None or c.label == label:
                    continue
                raise
            except Brk as b:
                if b.label is None or b.label == label:
                    break
                raise
        return ()

    def e_while(self, e, sc, label=None):
        while self.eval(e[1], sc):
            try:
                self.eval(e[2], sc)
            except Cont as c:
                if c.label is None or c.label == label:
                    continue
                raise
            except Brk as b:
                if b.label is None or b.label == label:
                    break
                raise
        return ()

    def e_loop(self, e, sc, label=None):
        while True:
            try:
                self.eval(e[1], sc)
            except Cont as c:
                if c.label is None or c.label == label:
                    continue
                raise
            except Brk as b:
                if b.label is None or b.label == label:
                    return b.v
                raise

    def e_return(self, e, sc):
        raise Ret(self.eval(e[1], sc) if e[1] is not None else ())

    def e_break(self, e, sc):
        raise Brk(self.eval(e[1], sc) if e[1] is not None else None, e[2] if len(e) > 2 else None)

    def e_continue(self, e, sc):
        raise Cont(e[1] if len(e) > 1 else None)

    def e_try(self, e, sc):
        v = self.eval(e[1], sc)
        if v is None:
            raise Ret(None)
        return v

    def e_closure(self, e, sc):
        _, params, body = e

        def fn(*args):
            inner = Scope(sc)
            if len(args) != len(params):
                raise RustError("closure arity")
            for p, a in zip(params, args):
                self.bind(p, a, inner)
            try:
                return self.eval(body, inner)
            except Ret as r:
                return r.v
        return fn

    def e_call(self, e, sc):
        fe = e[1]
        args = [self.eval(a, sc) for a in e[2]]
        if fe[0] == "path":
            path = fe[1]
            name = path[-1]
            if len(path) == 1:
                s = sc.lookup(name)
                if s is not None:
                    return s.vars[name](*args)
            if len(path) >= 2:
                key = f"{self._self_type(path[-2], sc)}::{name}"
                if key in self.builtins:
                    return self.builtins[key](*args)
                if key in self.mod.fns:
                    return self.call_fn(self.mod.fns[key], args)
            if name in self.mod.fns and (len(path) == 1 or path[-2] not in ("F", "Vec", "std", "core", "cmp")):
                return self.call_fn(self.mod.fns[name], args)
            if name == "Some" or name == "Ok":
                return args[0]
        f = self.eval(fe, sc)
        return f(*args)

    def e_mcall(self, e, sc):
        name = e[2]
        if name == "copy_from_slice" and e[1][0] == "index":
            # dst[a..b].copy_from_slice(src) writes through to dst
            arr = dv(self.eval(e[1][1], sc))
            i = self.eval(e[1][2], sc)
            src = list(dv(self.eval(e[3][0], sc)))
            if isinstance(i, RRange):
                lo = 0 if i.lo is None else i.lo
                hi = len(arr) if i.hi is None else (i.hi + 1 if i.inclusive else i.hi)
                if hi - lo != len(src):
                    raise RustError("copy_from_slice length mismatch")
                arr[lo:hi] = src
                return ()
        recv = self.eval(e[1], sc)
        args = [self.eval(a, sc) for a in e[3]]
        r = dv(recv)
        if isinstance(r, Struct):
            key = f"{r._name}::{name}"
            if key in self.builtins:
                return self.builtins[key](r, *args)
            if key in self.mod.fns:
                return self.call_fn(self.mod.fns[key], [r] + args)
        return method(recv, name, args)


def binop(op, a, b):
    if isinstance(a, Fe) or isinstance(b, Fe):
        if op == "+":
            return a + b
        if op == "-":
            return a - b
        if op == "*":
            return a * b
        if op == "/":
            return a / b
        if op == "==":
            return a == b
        if op == "!=":
            return not (a == b)
        raise RustError(f"field op {op}")
    if op == "+":
        return a + b
    if op == "-":
        return a - b
    if op == "*":
        return a * b
    if op == "/":
        if b == 0:
            raise RustError("integer division by zero")
        q = abs(a) // abs(b)
        return q if (a >= 0) == (b >= 0) else -q
    if op == "%":
        r = abs(a) % abs(b)
        return r if a >= 0 else -r
    if op == "<<":
        return a << b
    if op == ">>":
        return a >> b
    if op == "&":
        return a & b
    if op == "|":
        return a | b
    if op == "^":
        return a ^ b
    if op == "==":
        return a == b
    if op == "!=":
        return a != b
    if op == "<":
        return a < b
    if op == ">":
        return a > b
    if op == "<=":
        return a <= b
    if op == ">=":
        return a >= b
    raise RustError(f"op {op}")


def _f_from(x):
    if isinstance(x, bool):
        return Fe(int(x))
    if isinstance(x, Fe):
        return x
    if x < 0:
        return Fe(x)  # i64 -> F: the field's negation
    return Fe(x)


def _from_le(bs):
    bs = list(bs)
    return sum(int(b) << (8 * i) for i, b in enumerate(bs))


def _from_be(bs):
    bs = list(bs)
    return sum(int(b) << (8 * (len(bs) - 1 - i)) for i, b in enumerate(bs))


BUILTIN_PATHS = {
    "Lazy::new": lambda f: f(),
    "u64::from_le_bytes": _from_le,
    "u64::from_be_bytes": _from_be,
    "u32::from_le_bytes": _from_le,
    "u32::from_be_bytes": _from_be,
    "F::one": lambda: Fe(1),
    "F::zero": lambda: Fe(0),
    "F::from": _f_from,
    "Vec::new": lambda: [],
    "Vec::with_capacity": lambda n: [],
    "cmp::min": min,
    "cmp::max": max,
    "std::cmp::min": min,
    "std::cmp::max": max,
    "Some": lambda x: x,
    "Ok": lambda x: x,
    "u64::MAX": U64,
    "u32::MAX": 0xFFFFFFFF,
    "usize::MAX": U64,
    "MAX": None,
}


def _sum(xs):
    acc = None
    for x in xs:
        acc = x if acc is None else acc + x
    return Fe(0) if acc is None else acc


def method(recv, name, args):
    recv = dv(recv)
    if isinstance(recv, Fe):
        if name in ("square",):
            return recv * recv
        if name == "double":
            return recv + recv
        if name == "inverse":
            return None if recv.v == 0 else Fe(pow(recv.v, P - 2, P))
        if name == "is_zero":
            return recv.v == 0
        if name == "is_one":
            return recv.v == 1
        if name == "pow":
            e = args[0]
            e = e[0] if isinstance(e, list) else e
            return Fe(pow(recv.v, e, P))
        if name in ("clone", "to_owned", "unwrap", "expect"):
            return recv
        raise RustError(f"F.{name}")
    if isinstance(recv, RRange):
        if name == "contains":
            return recv.contains(args[0])
        return method(recv.items(), name, args)
    if isinstance(recv, bool):
        if name == "then":
            return args[0]() if recv else None
        if name in ("clone",):
            return recv
        raise RustError(f"bool.{name}")
    if isinstance(recv, int):
        if name == "saturating_sub":
            return max(0, recv - args[0])
        if name in ("wrapping_add",):
            return (recv + args[0]) & U64
        if name in ("wrapping_sub",):
            return (recv - args[0]) & U64
        if name in ("wrapping_mul",):
            return (recv * args[0]) & U64
        if name == "min":
            return min(recv, args[0])
        if name == "max":
            return max(recv, args[0])
        if name == "pow":
            return recv ** args[0]
        if name == "is_power_of_two":
            return recv > 0 and recv & (recv - 1) == 0
        if name == "trailing_zeros":
            return (recv & -recv).bit_length() - 1 if recv else 64
        if name == "count_ones":
            return bin(recv).count("1")
        if name == "div_ceil":
            return -(-recv // args[0])
        if name == "next_power_of_two":
            n = 1
            while n < recv:
                n <<= 1
            return n
        if name == "abs":
            return abs(recv)
        if name == "rem_euclid":
            return recv % abs(args[0])
        if name == "div_euclid":
            q = recv // abs(args[0])
            return q if args[0] > 0 else -q
        if name == "to_le_bytes":
            return [(recv >> (8 * i)) & 0xFF for i in range(8)]
        if name == "to_be_bytes":
            return [(recv >> (8 * (7 - i))) & 0xFF for i in range(8)]
        if name in ("clone",):
            return recv
        raise RustError(f"int.{name}")
    if isinstance(recv, Struct):
        if name == "clone":
            return recv.clone()
        if name in ("unwrap", "expect"):
            return recv
        raise RustError(f"struct.{name}")
    if isinstance(recv, tuple):
        recv = list(recv)
    if isinstance(recv, list):
        if name == "push":
            recv.append(args[0])
            return ()
        if name in ("extend", "extend_from_slice", "append"):
            recv.extend(list(args[0]))
            if name == "append":
                args[0].clear()
            return ()
        if name == "len":
            return len(recv)
        if name == "is_empty":
            return len(recv) == 0
        if name in ("iter", "into_iter", "iter_mut", "copied", "cloned", "collect", "to_vec", "as_slice",
                    "by_ref"):
            return list(recv)
        if name == "clone":
            return _clone(recv)
        if name == "map":
            return [args[0](x) for x in recv]
        if name == "filter":
            return [x for x in recv if args[0](x)]
        if name == "enumerate":
            return [(i, x) for i, x in enumerate(recv)]
        if name == "zip":
            return list(zip(recv, list(args[0]) if not isinstance(args[0], RRange) else args[0].items()))
        if name == "rev":
            return recv[::-1]
        if name == "sum":
            return _sum(recv)
        if name == "fold":
            acc = args[0]
            for x in recv:
                acc = args[1](acc, x)
            return acc
        if name == "all":
            return all(args[0](x) for x in recv)
        if name == "any":
            return any(args[0](x) for x in recv)
        if name == "skip":
            return recv[args[0]:]
        if name == "take":
            return recv[:args[0]]
        if name == "step_by":
            return recv[::args[0]]
        if name == "chain":
            return recv + list(args[0])
        if name == "last":
            return recv[-1] if recv else None
        if name == "first":
            return recv[0] if recv else None
        if name == "resize":
            n, v = args
            del recv[n:]
            recv.extend(_clone(v) for _ in range(n - len(recv)))
            return ()
        if name == "fill":
            for i in range(len(recv)):
                recv[i] = args[0]
            return ()
        if name == "copy_from_slice":
            recv[:] = list(args[0])
            return ()
        if name == "truncate":
            del recv[args[0]:]
            return ()
        if name == "chunks":
            k = args[0]
            return [recv[i:i + k] for i in range(0, len(recv), k)]
        if name == "contains":
            return args[0] in recv
        if name in ("unwrap", "expect", "try_into"):
            return recv
        if name == "get":
            i = args[0]
            return recv[i] if 0 <= i < len(recv) else None
        raise RustError(f"list.{name}")
    if recv is None and name in ("unwrap", "expect"):
        raise RustError("unwrap of None")
    if name in ("unwrap", "expect", "clone", "to_owned"):
        return recv
    raise RustError(f"method {name} on {type(recv).__name__}")
