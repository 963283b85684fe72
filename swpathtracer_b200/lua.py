"""A Lua 5.3 subset interpreter: enough of the language to run swpathtracer's scene scripts.

The reference renderer describes scenes in Lua (its lua_core/*.lua defines Camera{...},
Material{...}, Triangle{...} and friends, which fill the global table __RENDERER_ELEMENTS__; the
scripts under samples/ call them).  There is no Lua runtime here, so this module implements the part
of the language those scripts use:

  * values: nil, booleans, integers and floats (Lua 5.3 arithmetic: // and % floor, / always float),
    strings, tables (hash + array part with the border rule for #), functions and closures;
  * statements: local, assignment (multiple targets), calls, function / local function definitions
    (dotted names and a:b methods), if / elseif / else, numeric and generic for, while,
    repeat-until, do-end, return, break;
  * expressions with Lua's precedence and right-associative .. and ^, varargs, table constructors,
    call sugar f{...} and f"...";
  * the library functions the scripts reach: print, type, tostring, tonumber, pairs, ipairs, next,
    select, error, assert, require with package.path / package.loaded, math.*, os.exit / time /
    clock, string.format / rep / sub / len / upper / lower, table.insert / remove / concat / unpack.

Missing on purpose: metatables, coroutines, goto, integer bit operators, string patterns.
"""
import math
import os
import random as _random
import time as _time

# ------------------------------------------------------------------------------------------------
# lexer
# ------------------------------------------------------------------------------------------------

KEYWORDS = {"and", "break", "do", "else", "elseif", "end", "false", "for", "function", "goto", "if", "in",
            "local", "nil", "not", "or", "repeat", "return", "then", "true", "until", "while"}
SYMBOLS = ["...", "..", "==", "~=", "<=", ">=", "//", "::", "<<", ">>",
           "+", "-", "*", "/", "%", "^", "#", "&", "~", "|", "<", ">", "=", "(", ")", "{", "}", "[", "]",
           ";", ":", ",", "."]


class LuaError(Exception):
    """A Lua runtime or syntax error (the message carries the chunk name and line)."""


class LuaExit(Exception):
    """os.exit(code) from a script."""

    def __init__(self, code):
        super().__init__("os.exit(%r)" % (code,))
        self.code = code


def _long_bracket(src, i):
    """If src[i:] opens a long bracket [[ or [==[, return (level, index after the opener)."""
    if src[i] != "[":
        return None
    j = i + 1
    while j < len(src) and src[j] == "=":
        j += 1
    if j < len(src) and src[j] == "[":
        return j - i - 1, j + 1
    return None


def tokenize(src, chunk="?"):
    toks, i, line, n = [], 0, 1, len(src)
    if src.startswith("#"):                       # shebang line
        while i < n and src[i] != "\n":
            i += 1
    while i < n:
        c = src[i]
        if c == "\n":
            line += 1
            i += 1
            continue
        if c in " \t\r\f\v":
            i += 1
            continue
        if src.startswith("--", i):
            lb = _long_bracket(src, i + 2) if i + 2 < n else None
            if lb:
                close = "]" + "=" * lb[0] + "]"
                j = src.find(close, lb[1])
                if j < 0:
                    raise LuaError("%s:%d: unfinished long comment" % (chunk, line))
                line += src.count("\n", i, j)
                i = j + len(close)
            else:
                while i < n and src[i] != "\n":
                    i += 1
            continue
        if c.isalpha() or c == "_":
            j = i + 1
            while j < n and (src[j].isalnum() or src[j] == "_"):
                j += 1
            w = src[i:j]
            toks.append(("kw" if w in KEYWORDS else "name", w, line))
            i = j
            continue
        if c.isdigit() or (c == "." and i + 1 < n and src[i + 1].isdigit()):
            j = i
            if src.startswith(("0x", "0X"), i):
                j = i + 2
                while j < n and (src[j] in "0123456789abcdefABCDEF."):
                    j += 1
                text = src[i:j]
                val = int(text, 16) if "." not in text else float.fromhex(text)
            else:
                while j < n and (src[j].isdigit() or src[j] == "."):
                    j += 1
                if j < n and src[j] in "eE":
                    j += 1
                    if j < n and src[j] in "+-":
                        j += 1
                    while j < n and src[j].isdigit():
                        j += 1
                text = src[i:j]
                val = float(text) if any(ch in text for ch in ".eE") else int(text)
            toks.append(("number", val, line))
            i = j
            continue
        if c in "\"'":
            j, out = i + 1, []
            while True:
                if j >= n or src[j] == "\n":
                    raise LuaError("%s:%d: unfinished string" % (chunk, line))
                ch = src[j]
                if ch == c:
                    break
                if ch == "\\":
                    j += 1
                    e = src[j]
                    simple = {"n": "\n", "t": "\t", "r": "\r", "a": "\a", "b": "\b", "f": "\f", "v": "\v",
                              "\\": "\\", '"': '"', "'": "'", "\n": "\n"}
                    if e in simple:
                        out.append(simple[e])
                        j += 1
                    elif e.isdigit():
                        k = j
                        while k < n and k < j + 3 and src[k].isdigit():
                            k += 1
                        out.append(chr(int(src[j:k])))
                        j = k
                    elif e == "x":
                        out.append(chr(int(src[j + 1:j + 3], 16)))
                        j += 3
                    else:
                        raise LuaError("%s:%d: invalid escape \\%s" % (chunk, line, e))
                    continue
                out.append(ch)
                j += 1
            toks.append(("string", "".join(out), line))
            i = j + 1
            continue
        lb = _long_bracket(src, i)
        if lb:
            close = "]" + "=" * lb[0] + "]"
            j = src.find(close, lb[1])
            if j < 0:
                raise LuaError("%s:%d: unfinished long string" % (chunk, line))
            s = src[lb[1]:j]
            if s.startswith("\n"):
                s = s[1:]
            toks.append(("string", s, line))
            line += src.count("\n", i, j)
            i = j + len(close)
            continue
        for sym in SYMBOLS:
            if src.startswith(sym, i):
                toks.append(("op", sym, line))
                i += len(sym)
                break
        else:
            raise LuaError("%s:%d: unexpected symbol %r" % (chunk, line, c))
    toks.append(("eof", None, line))
    return toks


# ------------------------------------------------------------------------------------------------
# parser: tokens -> tuples
# ------------------------------------------------------------------------------------------------

BINARY_PRIORITY = {  # (left, right) binding power: the precedence order of the Lua 5.3 manual, 3.4.8
    "or": (1, 1), "and": (2, 2),
    "<": (3, 3), ">": (3, 3), "<=": (3, 3), ">=": (3, 3), "~=": (3, 3), "==": (3, 3),
    "|": (4, 4), "~": (5, 5), "&": (6, 6), "<<": (7, 7), ">>": (7, 7),
    "..": (9, 8), "+": (10, 10), "-": (10, 10),
    "*": (11, 11), "/": (11, 11), "//": (11, 11), "%": (11, 11),
    "^": (14, 13),
}
UNARY_PRIORITY = 12


class Parser:
    def __init__(self, src, chunk="?"):
        self.toks = tokenize(src, chunk)
        self.i = 0
        self.chunk = chunk

    # token helpers
    def peek(self, k=0):
        return self.toks[self.i + k]

    def error(self, msg):
        t = self.peek()
        raise LuaError("%s:%d: %s near %r" % (self.chunk, t[2], msg, t[1] if t[1] is not None else "<eof>"))

    def check(self, kind, value=None):
        t = self.peek()
        return t[0] == kind and (value is None or t[1] == value)

    def accept(self, kind, value=None):
        if self.check(kind, value):
            self.i += 1
            return True
        return False

    def expect(self, kind, value=None):
        if not self.check(kind, value):
            self.error("'%s' expected" % (value or kind))
        t = self.peek()
        self.i += 1
        return t

    def name(self):
        return self.expect("name")[1]

    # blocks and statements
    def parse(self):
        b = self.block()
        if not self.check("eof"):
            self.error("'<eof>' expected")
        return b

    def block_end(self):
        t = self.peek()
        return t[0] == "eof" or (t[0] == "kw" and t[1] in ("end", "else", "elseif", "until"))

    def block(self):
        stmts = []
        while not self.block_end():
            if self.check("kw", "return"):
                line = self.peek()[2]
                self.i += 1
                exprs = [] if (self.block_end() or self.check("op", ";")) else self.exprlist()
                self.accept("op", ";")
                stmts.append(("Return", exprs, line))
                break
            s = self.statement()
            if s is not None:
                stmts.append(s)
        return ("Block", stmts)

    def statement(self):
        t = self.peek()
        line = t[2]
        if self.accept("op", ";"):
            return None
        if t[0] == "kw":
            w = t[1]
            if w == "if":
                self.i += 1
                arms = [(self.expr(), self._then_block())]
                orelse = None
                while True:
                    if self.accept("kw", "elseif"):
                        arms.append((self.expr(), self._then_block()))
                    elif self.accept("kw", "else"):
                        orelse = self.block()
                        self.expect("kw", "end")
                        break
                    else:
                        self.expect("kw", "end")
                        break
                return ("If", arms, orelse, line)
            if w == "while":
                self.i += 1
                cond = self.expr()
                self.expect("kw", "do")
                body = self.block()
                self.expect("kw", "end")
                return ("While", cond, body, line)
            if w == "do":
                self.i += 1
                body = self.block()
                self.expect("kw", "end")
                return ("Do", body, line)
            if w == "for":
                self.i += 1
                n1 = self.name()
                if self.accept("op", "="):
                    start = self.expr()
                    self.expect("op", ",")
                    stop = self.expr()
                    step = self.expr() if self.accept("op", ",") else None
                    self.expect("kw", "do")
                    body = self.block()
                    self.expect("kw", "end")
                    return ("NumFor", n1, start, stop, step, body, line)
                names = [n1]
                while self.accept("op", ","):
                    names.append(self.name())
                self.expect("kw", "in")
                exprs = self.exprlist()
                self.expect("kw", "do")
                body = self.block()
                self.expect("kw", "end")
                return ("GenFor", names, exprs, body, line)
            if w == "repeat":
                self.i += 1
                body = self.block()
                self.expect("kw", "until")
                return ("Repeat", body, self.expr(), line)
            if w == "function":
                self.i += 1
                path = [self.name()]
                method = None
                while self.accept("op", "."):
                    path.append(self.name())
                if self.accept("op", ":"):
                    method = self.name()
                f = self.funcbody(method is not None, line)
                return ("FunctionStat", path, method, f, line)
            if w == "local":
                self.i += 1
                if self.accept("kw", "function"):
                    n = self.name()
                    return ("LocalFunction", n, self.funcbody(False, line), line)
                names = [self.name()]
                while self.accept("op", ","):
                    names.append(self.name())
                exprs = self.exprlist() if self.accept("op", "=") else []
                return ("Local", names, exprs, line)
            if w == "break":
                self.i += 1
                return ("Break", line)
            if w == "goto":
                self.error("goto is not supported")
        # expression statement: a call or an assignment
        e = self.suffixedexp()
        if self.check("op", "=") or self.check("op", ","):
            targets = [e]
            while self.accept("op", ","):
                targets.append(self.suffixedexp())
            self.expect("op", "=")
            for tg in targets:
                if tg[0] not in ("Name", "Index"):
                    self.error("cannot assign to this expression")
            return ("Assign", targets, self.exprlist(), line)
        if e[0] not in ("Call", "Method"):
            self.error("syntax error")
        return ("CallStat", e, line)

    def _then_block(self):
        self.expect("kw", "then")
        return self.block()

    def funcbody(self, is_method, line):
        self.expect("op", "(")
        params = ["self"] if is_method else []
        vararg = False
        if not self.check("op", ")"):
            while True:
                if self.accept("op", "..."):
                    vararg = True
                    break
                params.append(self.name())
                if not self.accept("op", ","):
                    break
        self.expect("op", ")")
        body = self.block()
        self.expect("kw", "end")
        return ("Func", params, vararg, body, line)

    # expressions
    def exprlist(self):
        es = [self.expr()]
        while self.accept("op", ","):
            es.append(self.expr())
        return es

    def expr(self, limit=0):
        t = self.peek()
        if (t[0] == "kw" and t[1] == "not") or (t[0] == "op" and t[1] in ("-", "#", "~")):
            self.i += 1
            left = ("Un", t[1], self.expr(UNARY_PRIORITY), t[2])
        else:
            left = self.simpleexp()
        while True:
            t = self.peek()
            op = t[1] if t[0] in ("op", "kw") else None
            if op not in BINARY_PRIORITY or BINARY_PRIORITY[op][0] <= limit:
                return left
            self.i += 1
            right = self.expr(BINARY_PRIORITY[op][1])
            if op == "and":
                left = ("And", left, right)
            elif op == "or":
                left = ("Or", left, right)
            else:
                left = ("Bin", op, left, right, t[2])

    def simpleexp(self):
        t = self.peek()
        if t[0] == "number":
            self.i += 1
            return ("Const", t[1])
        if t[0] == "string":
            self.i += 1
            return ("Const", t[1])
        if t[0] == "kw":
            if t[1] == "nil":
                self.i += 1
                return ("Const", None)
            if t[1] == "true":
                self.i += 1
                return ("Const", True)
            if t[1] == "false":
                self.i += 1
                return ("Const", False)
            if t[1] == "function":
                self.i += 1
                return self.funcbody(False, t[2])
        if self.check("op", "..."):
            self.i += 1
            return ("Vararg",)
        if self.check("op", "{"):
            return self.table()
        return self.suffixedexp()

    def primaryexp(self):
        t = self.peek()
        if t[0] == "name":
            self.i += 1
            return ("Name", t[1], t[2])
        if self.accept("op", "("):
            e = self.expr()
            self.expect("op", ")")
            return ("Paren", e)
        self.error("unexpected symbol")

    def suffixedexp(self):
        e = self.primaryexp()
        while True:
            t = self.peek()
            if self.accept("op", "."):
                e = ("Index", e, ("Const", self.name()), t[2])
            elif self.accept("op", "["):
                k = self.expr()
                self.expect("op", "]")
                e = ("Index", e, k, t[2])
            elif self.accept("op", ":"):
                m = self.name()
                e = ("Method", e, m, self.callargs(), t[2])
            elif self.check("op", "(") or self.check("op", "{") or self.check("string"):
                e = ("Call", e, self.callargs(), t[2])
            else:
                return e

    def callargs(self):
        if self.check("string"):
            return [("Const", self.expect("string")[1])]
        if self.check("op", "{"):
            return [self.table()]
        self.expect("op", "(")
        if self.accept("op", ")"):
            return []
        args = self.exprlist()
        self.expect("op", ")")
        return args

    def table(self):
        self.expect("op", "{")
        items = []   # (key expr or None for positional, value expr)
        while not self.check("op", "}"):
            if self.check("op", "["):
                self.i += 1
                k = self.expr()
                self.expect("op", "]")
                self.expect("op", "=")
                items.append((k, self.expr()))
            elif self.check("name") and self.peek(1)[0] == "op" and self.peek(1)[1] == "=":
                k = ("Const", self.name())
                self.i += 1
                items.append((k, self.expr()))
            else:
                items.append((None, self.expr()))
            if not (self.accept("op", ",") or self.accept("op", ";")):
                break
        self.expect("op", "}")
        return ("Table", items)


# ------------------------------------------------------------------------------------------------
# values
# ------------------------------------------------------------------------------------------------

class LuaTable:
    """A Lua table: one dict; integral float keys are stored as ints, as Lua normalises them."""
    __slots__ = ("d",)

    def __init__(self, items=None):
        self.d = {}
        if items:
            for k, v in items:
                self[k] = v

    @staticmethod
    def _key(k):
        if isinstance(k, float) and k.is_integer():
            return int(k)
        return k

    def __getitem__(self, k):
        return self.d.get(self._key(k))

    def __setitem__(self, k, v):
        if k is None:
            raise LuaError("table index is nil")
        if isinstance(k, float) and k != k:
            raise LuaError("table index is NaN")
        k = self._key(k)
        if v is None:
            self.d.pop(k, None)
        else:
            self.d[k] = v

    def length(self):
        """A border: n with t[n] ~= nil and t[n+1] == nil (the largest when the array part is dense)."""
        n = 0
        while (n + 1) in self.d:
            n += 1
        return n

    def array(self):
        return [self.d[i] for i in range(1, self.length() + 1)]

    def get(self, k, default=None):
        v = self[k]
        return default if v is None else v


class LuaFunction:
    __slots__ = ("params", "vararg", "body", "scope", "name")

    def __init__(self, params, vararg, body, scope, name="?"):
        self.params, self.vararg, self.body, self.scope, self.name = params, vararg, body, scope, name


class _Break(Exception):
    pass


class _Return(Exception):
    def __init__(self, values):
        self.values = values


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


def lua_type(v):
    if v is None:
        return "nil"
    if isinstance(v, bool):
        return "boolean"
    if isinstance(v, (int, float)):
        return "number"
    if isinstance(v, str):
        return "string"
    if isinstance(v, LuaTable):
        return "table"
    return "function"


def truthy(v):
    return v is not None and v is not False


def tostr(v):
    if v is None:
        return "nil"
    if v is True:
        return "true"
    if v is False:
        return "false"
    if isinstance(v, int):
        return str(v)
    if isinstance(v, float):
        if v == math.inf:
            return "inf"
        if v == -math.inf:
            return "-inf"
        if v != v:
            return "nan"
        if v.is_integer() and abs(v) < 1e16:
            return "%.1f" % v
        return "%.14g" % v
    if isinstance(v, str):
        return v
    if isinstance(v, LuaTable):
        return "table: 0x%08x" % (id(v) & 0xFFFFFFFF)
    return "function: 0x%08x" % (id(v) & 0xFFFFFFFF)


def tonum(v):
    if isinstance(v, bool):
        return None
    if isinstance(v, (int, float)):
        return v
    if isinstance(v, str):
        t = v.strip()
        try:
            if t.lower().startswith(("0x", "-0x")):
                return int(t, 16)
            return int(t) if t.lstrip("+-").isdigit() else float(t)
        except ValueError:
            return None
    return None


def _arith_operand(v, op):
    n = tonum(v) if isinstance(v, str) else v
    if isinstance(n, bool) or not isinstance(n, (int, float)):
        raise LuaError("attempt to perform arithmetic (%s) on a %s value" % (op, lua_type(v)))
    return n


def arith(op, a, b):
    x, y = _arith_operand(a, op), _arith_operand(b, op)
    if op == "+":
        return x + y
    if op == "-":
        return x - y
    if op == "*":
        return x * y
    if op == "/":
        y = float(y)
        if y == 0.0:
            x = float(x)
            return math.copysign(math.inf, x) * math.copysign(1.0, y) if x != 0 else math.nan
        return float(x) / y
    if op == "//":
        if isinstance(x, int) and isinstance(y, int):
            if y == 0:
                raise LuaError("attempt to perform 'n//0'")
            return x // y
        return float(math.floor(float(x) / float(y))) if y != 0 else arith("/", x, y)
    if op == "%":
        if isinstance(x, int) and isinstance(y, int):
            if y == 0:
                raise LuaError("attempt to perform 'n%%0'")
            return x % y
        if y == 0:
            return math.nan
        r = math.fmod(float(x), float(y))
        return r + y if r != 0 and (r < 0) != (y < 0) else r
    if op == "^":
        return float(x) ** float(y)
    raise LuaError("unknown operator " + op)


def compare(op, a, b):
    if isinstance(a, bool) or isinstance(b, bool) or lua_type(a) != lua_type(b) or \
            lua_type(a) not in ("number", "string"):
        if op in ("==", "~="):
            eq = (a is b) or (type(a) == type(b) and a == b and not isinstance(a, (LuaTable, LuaFunction)))
            return eq if op == "==" else not eq
        raise LuaError("attempt to compare %s with %s" % (lua_type(a), lua_type(b)))
    if op == "==":
        return a == b
    if op == "~=":
        return a != b
    if op == "<":
        return a < b
    if op == "<=":
        return a <= b
    if op == ">":
        return a > b
    return a >= b


# ------------------------------------------------------------------------------------------------
# interpreter
# ------------------------------------------------------------------------------------------------

class Interpreter:
    """Runs Lua chunks against one global table (`G`)."""

    def __init__(self, search_dirs=(), seed=None):
        self.G = LuaTable()
        self.search_dirs = list(search_dirs)   # base directories for relative package.path entries
        self.rng = _random.Random(seed)
        self.output = []                       # what print() wrote, one string per call
        self._install_stdlib()

    # ---- running chunks ----------------------------------------------------------------------
    def run_string(self, src, chunk="=(string)"):
        tree = Parser(src, chunk).parse()
        return self.call(LuaFunction([], True, tree, None, chunk), [])

    def run_file(self, path):
        path = os.path.abspath(path)
        d = os.path.dirname(path)
        if d not in self.search_dirs:
            self.search_dirs.append(d)
        with open(path) as f:
            return self.run_string(f.read(), os.path.basename(path))

    # ---- calls ------------------------------------------------------------------------------
    def call(self, f, args):
        if isinstance(f, LuaFunction):
            scope = Scope(f.scope)
            n = len(f.params)
            for i, p in enumerate(f.params):
                scope.vars[p] = args[i] if i < len(args) else None
            varargs = list(args[n:]) if f.vararg else []
            try:
                self.exec_block(f.body, scope, varargs)
            except _Return as r:
                return r.values
            return []
        if callable(f):
            r = f(*args)
            if r is None:
                return []
            return list(r) if isinstance(r, (list, tuple)) else [r]
        raise LuaError("attempt to call a %s value" % lua_type(f))

    # ---- statements -------------------------------------------------------------------------
    def exec_block(self, block, scope, varargs):
        for st in block[1]:
            self.exec_stmt(st, scope, varargs)

    def exec_stmt(self, st, scope, va):
        k = st[0]
        try:
            if k == "Local":
                vals = self.eval_list(st[2], scope, va)
                for i, name in enumerate(st[1]):
                    scope.vars[name] = vals[i] if i < len(vals) else None
            elif k == "Assign":
                vals = self.eval_list(st[2], scope, va)
                for i, tg in enumerate(st[1]):
                    self.assign(tg, vals[i] if i < len(vals) else None, scope, va)
            elif k == "CallStat":
                self.eval_call(st[1], scope, va)
            elif k == "If":
                for cond, body in st[1]:
                    if truthy(self.eval(cond, scope, va)):
                        self.exec_block(body, Scope(scope), va)
                        return
                if st[2] is not None:
                    self.exec_block(st[2], Scope(scope), va)
            elif k == "NumFor":
                start = _arith_operand(self.eval(st[2], scope, va), "for")
                stop = _arith_operand(self.eval(st[3], scope, va), "for")
                step = _arith_operand(self.eval(st[4], scope, va), "for") if st[4] is not None else 1
                if step == 0:
                    raise LuaError("'for' step is zero")
                if not (isinstance(start, int) and isinstance(step, int)):
                    start, stop, step = float(start), float(stop), float(step)
                i = start
                try:
                    while (i <= stop) if step > 0 else (i >= stop):
                        s = Scope(scope)
                        s.vars[st[1]] = i
                        self.exec_block(st[5], s, va)
                        i += step
                except _Break:
                    pass
            elif k == "GenFor":
                vals = self.eval_list(st[2], scope, va) + [None, None, None]
                f, state, ctl = vals[0], vals[1], vals[2]
                try:
                    while True:
                        rs = self.call(f, [state, ctl])
                        if not rs or rs[0] is None:
                            break
                        ctl = rs[0]
                        s = Scope(scope)
                        for i, name in enumerate(st[1]):
                            s.vars[name] = rs[i] if i < len(rs) else None
                        self.exec_block(st[3], s, va)
                except _Break:
                    pass
            elif k == "While":
                try:
                    while truthy(self.eval(st[1], scope, va)):
                        self.exec_block(st[2], Scope(scope), va)
                except _Break:
                    pass
            elif k == "Repeat":
                try:
                    while True:
                        s = Scope(scope)
                        self.exec_block(st[1], s, va)
                        if truthy(self.eval(st[2], s, va)):
                            break
                except _Break:
                    pass
            elif k == "Do":
                self.exec_block(st[1], Scope(scope), va)
            elif k == "FunctionStat":
                path, method, fn = st[1], st[2], st[3]
                f = LuaFunction(fn[1], fn[2], fn[3], scope, ".".join(path) + (":" + method if method else ""))
                if len(path) == 1 and method is None:
                    self.assign(("Name", path[0], st[4]), f, scope, va)
                else:
                    obj = self.eval(("Name", path[0], st[4]), scope, va)
                    for p in (path[1:] if method else path[1:-1]):
                        obj = self.index(obj, p)
                    self.setindex(obj, method if method else path[-1], f)
            elif k == "LocalFunction":
                fn = st[2]
                scope.vars[st[1]] = None
                scope.vars[st[1]] = LuaFunction(fn[1], fn[2], fn[3], scope, st[1])
            elif k == "Return":
                raise _Return(self.eval_list(st[1], scope, va))
            elif k == "Break":
                raise _Break()
            else:
                raise LuaError("unknown statement " + k)
        except LuaError as e:
            msg = str(e)
            if not msg.startswith("line "):
                raise LuaError("line %d: %s" % (st[-1], msg)) from None
            raise

    def assign(self, tg, v, scope, va):
        if tg[0] == "Name":
            s = scope.lookup(tg[1]) if scope is not None else None
            if s is not None:
                s.vars[tg[1]] = v
            else:
                self.G[tg[1]] = v
        else:
            self.setindex(self.eval(tg[1], scope, va), self.eval(tg[2], scope, va), v)

    # ---- expressions ------------------------------------------------------------------------
    def index(self, obj, key):
        if isinstance(obj, LuaTable):
            return obj[key]
        if isinstance(obj, str):
            return self.G["string"][key]
        raise LuaError("attempt to index a %s value (key %r)" % (lua_type(obj), key))

    def setindex(self, obj, key, v):
        if not isinstance(obj, LuaTable):
            raise LuaError("attempt to index a %s value (key %r)" % (lua_type(obj), key))
        obj[key] = v

    def eval_list(self, exprs, scope, va):
        out = []
        for i, e in enumerate(exprs):
            if i == len(exprs) - 1 and e[0] in ("Call", "Method", "Vararg"):
                out.extend(self.eval_multi(e, scope, va))
            else:
                out.append(self.eval(e, scope, va))
        return out

    def eval_multi(self, e, scope, va):
        if e[0] == "Vararg":
            return list(va)
        return self.eval_call(e, scope, va)

    def eval_call(self, e, scope, va):
        if e[0] == "Method":
            obj = self.eval(e[1], scope, va)
            f = self.index(obj, e[2])
            return self.call(f, [obj] + self.eval_list(e[3], scope, va))
        f = self.eval(e[1], scope, va)
        return self.call(f, self.eval_list(e[2], scope, va))

    def eval(self, e, scope, va):
        k = e[0]
        if k == "Const":
            return e[1]
        if k == "Name":
            s = scope.lookup(e[1]) if scope is not None else None
            return s.vars[e[1]] if s is not None else self.G[e[1]]
        if k == "Index":
            return self.index(self.eval(e[1], scope, va), self.eval(e[2], scope, va))
        if k in ("Call", "Method"):
            r = self.eval_call(e, scope, va)
            return r[0] if r else None
        if k == "Bin":
            op = e[1]
            a, b = self.eval(e[2], scope, va), self.eval(e[3], scope, va)
            if op in ("==", "~=", "<", "<=", ">", ">="):
                return compare(op, a, b)
            if op == "..":
                for x in (a, b):
                    if not isinstance(x, (str, int, float)) or isinstance(x, bool):
                        raise LuaError("attempt to concatenate a %s value" % lua_type(x))
                return tostr(a) + tostr(b)
            return arith(op, a, b)
        if k == "And":
            a = self.eval(e[1], scope, va)
            return self.eval(e[2], scope, va) if truthy(a) else a
        if k == "Or":
            a = self.eval(e[1], scope, va)
            return a if truthy(a) else self.eval(e[2], scope, va)
        if k == "Un":
            op, v = e[1], self.eval(e[2], scope, va)
            if op == "not":
                return not truthy(v)
            if op == "-":
                return -_arith_operand(v, "unm")
            if op == "#":
                if isinstance(v, str):
                    return len(v)
                if isinstance(v, LuaTable):
                    return v.length()
                raise LuaError("attempt to get length of a %s value" % lua_type(v))
            raise LuaError("unsupported unary operator " + op)
        if k == "Paren":
            return self.eval(e[1], scope, va)
        if k == "Vararg":
            return va[0] if va else None
        if k == "Func":
            return LuaFunction(e[1], e[2], e[3], scope)
        if k == "Table":
            t = LuaTable()
            n = 0
            items = e[1]
            for i, (key, val) in enumerate(items):
                if key is None:
                    if i == len(items) - 1 and val[0] in ("Call", "Method", "Vararg"):
                        for v in self.eval_multi(val, scope, va):
                            n += 1
                            t[n] = v
                    else:
                        n += 1
                        t[n] = self.eval(val, scope, va)
                else:
                    t[self.eval(key, scope, va)] = self.eval(val, scope, va)
            return t
        raise LuaError("unknown expression " + k)

    # ---- standard library -------------------------------------------------------------------
    def _install_stdlib(self):
        G = self.G
        G["_G"] = G
        G["_VERSION"] = "Lua 5.3"

        def _print(*a):
            line = "\t".join(tostr(x) for x in a)
            self.output.append(line)
        G["print"] = _print
        G["type"] = lambda v=None: lua_type(v)
        G["tostring"] = lambda v=None: tostr(v)

        def _tonumber(v=None, base=None):
            if base is None:
                return tonum(v)
            try:
                return int(str(v).strip(), int(base))
            except ValueError:
                return None
        G["tonumber"] = _tonumber

        def _next(t, k=None):
            keys = list(t.d.keys())
            if k is None:
                i = 0
            else:
                k = LuaTable._key(k)
                if k not in t.d:
                    raise LuaError("invalid key to 'next'")
                i = keys.index(k) + 1
            if i >= len(keys):
                return [None]
            return [keys[i], t.d[keys[i]]]
        G["next"] = _next

        def _pairs(t):
            if not isinstance(t, LuaTable):
                raise LuaError("bad argument #1 to 'pairs' (table expected, got %s)" % lua_type(t))
            snapshot = list(t.d.items())
            it = iter(snapshot)

            def step(_s, _c):
                for kk, vv in it:
                    if t.d.get(kk) is not None:
                        return [kk, vv]
                return [None]
            return [step, t, None]
        G["pairs"] = _pairs

        def _ipairs(t):
            def step(_s, i):
                v = t[i + 1]
                return [None] if v is None else [i + 1, v]
            return [step, t, 0]
        G["ipairs"] = _ipairs

        def _select(n, *a):
            if n == "#":
                return len(a)
            n = int(n)
            return list(a[n - 1:]) if n > 0 else list(a[n:])
        G["select"] = _select

        def _error(msg=None, level=1):
            raise LuaError(tostr(msg))
        G["error"] = _error

        def _assert(v=None, msg="assertion failed!", *rest):
            if not truthy(v):
                raise LuaError(tostr(msg))
            return [v, msg] + list(rest)
        G["assert"] = _assert

        def _unpack(t, i=1, j=None):
            j = t.length() if j is None else int(j)
            return [t[k] for k in range(int(i), j + 1)]
        G["unpack"] = _unpack

        # package / require
        package = LuaTable()
        package["path"] = "./?.lua;./?/init.lua"
        package["loaded"] = LuaTable()
        G["package"] = package

        def _require(name):
            loaded = package["loaded"]
            if loaded[name] is not None:
                return loaded[name]
            tried = []
            for templ in tostr(package["path"]).split(";"):
                if not templ:
                    continue
                cand = templ.replace("?", name.replace(".", "/"))
                paths = [cand] if os.path.isabs(cand) else [os.path.join(d, cand) for d in [os.getcwd()] + self.search_dirs]
                for pth in paths:
                    tried.append(pth)
                    if os.path.isfile(pth):
                        with open(pth) as f:
                            src = f.read()
                        loaded[name] = True   # a module that requires itself back sees it as loaded
                        r = self.call(LuaFunction([], True, Parser(src, os.path.basename(pth)).parse(), None, name),
                                      [name])
                        loaded[name] = r[0] if r and r[0] is not None else True
                        return loaded[name]
            raise LuaError("module '%s' not found (tried %s)" % (name, ", ".join(tried)))
        G["require"] = _require

        # math
        m = LuaTable()
        m["huge"] = math.inf
        m["pi"] = math.pi
        m["maxinteger"] = 2 ** 63 - 1
        m["mininteger"] = -2 ** 63
        for fname in ("sqrt", "sin", "cos", "tan", "asin", "acos", "atan", "exp"):
            m[fname] = (lambda fn: lambda x: fn(float(_arith_operand(x, fn.__name__))))(getattr(math, fname))
        m["atan"] = lambda y, x=1.0: math.atan2(float(y), float(x))
        m["log"] = lambda x, b=None: math.log(float(x)) if b is None else math.log(float(x), float(b))
        m["floor"] = lambda x: int(math.floor(x)) if math.isfinite(x) else x
        m["ceil"] = lambda x: int(math.ceil(x)) if math.isfinite(x) else x
        m["abs"] = lambda x: abs(x)
        m["fmod"] = lambda a, b: math.fmod(a, b)
        m["modf"] = lambda x: [float(math.trunc(x)), x - math.trunc(x)]
        m["min"] = lambda *a: min(a)
        m["max"] = lambda *a: max(a)
        m["tointeger"] = lambda x: int(x) if isinstance(x, (int, float)) and float(x).is_integer() else None
        m["type"] = lambda x=None: ("integer" if isinstance(x, int) else "float") \
            if isinstance(x, (int, float)) and not isinstance(x, bool) else None

        def _random_fn(a=None, b=None):
            if a is None:
                return self.rng.random()
            lo, hi = (1, int(a)) if b is None else (int(a), int(b))
            if lo > hi:
                raise LuaError("bad argument to 'random' (interval is empty)")
            return self.rng.randint(lo, hi)
        m["random"] = _random_fn
        m["randomseed"] = lambda x=None: self.rng.seed(x)
        G["math"] = m

        # os
        o = LuaTable()

        def _exit(code=None, close=None):
            raise LuaExit(code)
        o["exit"] = _exit
        o["time"] = lambda t=None: int(_time.time())
        o["clock"] = lambda: _time.process_time()
        o["getenv"] = lambda k: os.environ.get(k)
        G["os"] = o

        # string
        st = LuaTable()

        def _format(fmt, *a):
            out, ai, i = [], 0, 0
            while i < len(fmt):
                c = fmt[i]
                if c != "%":
                    out.append(c)
                    i += 1
                    continue
                j = i + 1
                while j < len(fmt) and fmt[j] in "-+ #0123456789.":
                    j += 1
                spec, conv = fmt[i:j], fmt[j]
                i = j + 1
                if conv == "%":
                    out.append("%")
                    continue
                v = a[ai]
                ai += 1
                if conv in "di":
                    out.append((spec + "d") % int(v))
                elif conv in "feEgGxXoc":
                    out.append((spec + conv) % (v if conv not in "xXoc" else int(v)))
                elif conv == "s":
                    out.append((spec + "s") % tostr(v))
                elif conv == "q":
                    out.append('"%s"' % tostr(v).replace("\\", "\\\\").replace('"', '\\"'))
                else:
                    raise LuaError("invalid conversion '%%%s' to 'format'" % conv)
            return "".join(out)
        st["format"] = _format
        st["rep"] = lambda s, n, sep="": sep.join([s] * int(n))
        st["len"] = lambda s: len(s)
        st["upper"] = lambda s: s.upper()
        st["lower"] = lambda s: s.lower()
        st["reverse"] = lambda s: s[::-1]

        def _sub(s, i=1, j=-1):
            n = len(s)
            i, j = int(i), int(j)
            if i < 0:
                i = max(n + i + 1, 1)
            elif i == 0:
                i = 1
            if j < 0:
                j = n + j + 1
            elif j > n:
                j = n
            return s[i - 1:j] if i <= j else ""
        st["sub"] = _sub
        G["string"] = st

        # table
        tb = LuaTable()

        def _insert(t, *a):
            if len(a) == 1:
                t[t.length() + 1] = a[0]
            else:
                pos, v = int(a[0]), a[1]
                n = t.length()
                for k in range(n, pos - 1, -1):
                    t[k + 1] = t[k]
                t[pos] = v
        tb["insert"] = _insert

        def _remove(t, pos=None):
            n = t.length()
            pos = n if pos is None else int(pos)
            v = t[pos]
            for k in range(pos, n):
                t[k] = t[k + 1]
            t[n] = None
            return v
        tb["remove"] = _remove
        tb["concat"] = lambda t, sep="", i=1, j=None: sep.join(
            tostr(t[k]) for k in range(int(i), (t.length() if j is None else int(j)) + 1))
        tb["unpack"] = _unpack
        G["table"] = tb


def run(path, search_dirs=(), seed=None):
    """Runs a Lua file; returns the interpreter (its globals hold what the script built)."""
    it = Interpreter(search_dirs, seed)
    it.run_file(path)
    return it
