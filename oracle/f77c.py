#!/usr/bin/env python3
"""Fortran-77 subset -> C translator: the recipe that builds the oracle reference.

TEST INFRASTRUCTURE ONLY.  Nothing in the product imports or runs this file.

The SPR library is Fortran-77 and this image has no Fortran compiler.  To run
the reference's own code anyway (as the pinned oracle and as the CPU
baseline), this script translates the SPR source files *mechanically* from
where they lie in the reference checkout into one C file under
``oracle/_ref/`` (git-ignored), which ``oracle/Makefile`` compiles with gcc
into ``oracle/_ref/libsprref.so``.  No reference source is copied into the
repository: only this translator is committed, and its output never is.

The translation keeps the Fortran semantics that matter for bit-exact
results:

* every INTEGER/LOGICAL is the default integer kind of the I8 build
  (``-fdefault-integer-8``), i.e. ``int64_t`` (``-DFINT=int32_t`` gives the
  I4 build); ``INTEGER(kind=i8)`` is always 64-bit;
* all arguments are passed by reference (constants and expressions through
  C99 compound-literal temporaries), arrays are column-major with their
  declared lower bounds, adjustable extents are evaluated on entry;
* DO loops evaluate their bounds once and leave the loop variable at
  ``start + trips*step``; labelled DO terminals (shared ones included),
  block IF, logical IF, GOTO, computed GOTO and arithmetic IF map onto C
  control flow with ``goto``;
* expression evaluation order and parenthesisation are kept as written
  (the output is compiled with ``-ffp-contract=off``, so no FMA is formed);
  single-precision literals stay ``float``; ``**`` uses gcc's ``powi``
  like gfortran does;
* WRITE/FORMAT/PRINT statements are dropped (message text is not part of
  the numeric contract; the error codes they accompany are kept).

Only the constructs used by the SPR files the oracle needs are supported;
anything else raises ``F77Error`` with the file and line.
"""
import os
import re
import sys


class F77Error(Exception):
    pass


# --------------------------------------------------------------------------
# Source reading (fixed form, cpp conditionals, continuation lines)
# --------------------------------------------------------------------------

def _pp_eval(expr, defines):
    expr = re.sub(r'defined\s*\(\s*(\w+)\s*\)',
                  lambda m: '1' if m.group(1) in defines else '0', expr)
    expr = re.sub(r'[A-Za-z_]\w*',
                  lambda m: str(defines.get(m.group(0), 0)), expr)
    expr = expr.replace('&&', ' and ').replace('||', ' or ').replace('!', ' not ')
    expr = expr.replace(' not =', '!=')
    if not re.fullmatch(r'[\d\s()<>=!andortn]*', expr):
        raise F77Error('cannot evaluate #if ' + expr)
    return bool(eval(expr))


_UNIT_HDR = re.compile(r'^ {6}\s*(?:(?:INTEGER|DOUBLE\s*PRECISION|REAL|LOGICAL)(?:\*\d+|\(\s*kind\s*=\s*\w+\s*\))?\s+)?'
                       r'(?:SUBROUTINE|FUNCTION)\s+(\w+)', re.I)
_UNIT_END = re.compile(r'^ {6}\s*END\s*$', re.I)


def _pick_units(raw_lines, keep):
    """Blank out every line outside the program units named in `keep` (a
    source file of many routines of which only a few are needed; line numbers
    are kept for the messages)."""
    out, inside = [], False
    for raw in raw_lines:
        m = _UNIT_HDR.match(raw)
        if m and not inside:
            inside = m.group(1).upper() in keep
        out.append(raw if inside else '')
        if inside and _UNIT_END.match(raw):
            inside = False
    return out


def read_statements(path, defines=None, keep=None):
    """Return [(label, text, 'file:line')] with continuations joined; with
    `keep`, only the named program units of the file."""
    defines = defines or {}
    out = []
    active = []                      # stack of (parent_active, this_active)
    with open(path, encoding='latin-1') as fh:
        raw_lines = fh.read().split('\n')
    if keep:
        raw_lines = _pick_units(raw_lines, keep)
    for ln, raw in enumerate(raw_lines, 1):
        raw = raw.rstrip('\r')
        if raw.startswith('#'):
            d = raw[1:].strip()
            on = all(a for a in active)
            if d.startswith('ifdef'):
                active.append(d.split()[1] in defines)
            elif d.startswith('ifndef'):
                active.append(d.split()[1] not in defines)
            elif d.startswith('if'):
                active.append(_pp_eval(d[2:], defines))
            elif d.startswith('else'):
                active[-1] = not active[-1]
            elif d.startswith('endif'):
                active.pop()
            else:
                raise F77Error('%s:%d unsupported directive %s' % (path, ln, raw))
            del on
            continue
        if not all(active):
            continue
        if not raw.strip():
            continue
        if raw[0] in 'Cc*!':
            continue
        line = raw.expandtabs(6)[:72]
        where = '%s:%d' % (os.path.basename(path), ln)
        if len(line) > 5 and line[5] not in ' 0' and not line[:5].strip():
            if not out:
                raise F77Error(where + ' continuation without statement')
            lab, txt, w = out[-1]
            out[-1] = (lab, txt + line[6:], w)
            continue
        label = line[:5].strip()
        if label and not label.isdigit():
            # free-form line starting in column 1 (e.g. an include file)
            label, body = '', line
        else:
            body = line[6:]
        out.append((label, body, where))
    # strip inline comments outside strings
    res = []
    for lab, txt, w in out:
        res.append((lab, _strip_inline_comment(txt), w))
    return res


def _strip_inline_comment(txt):
    inq = False
    for i, ch in enumerate(txt):
        if ch == "'":
            inq = not inq
        elif ch == '!' and not inq:
            return txt[:i]
    return txt


def normalise(txt):
    """Upper-case and drop blanks outside strings; strings become $n$."""
    strings = []
    buf = []
    i = 0
    while i < len(txt):
        ch = txt[i]
        if ch == "'":
            j = i + 1
            s = []
            while True:
                if j >= len(txt):
                    raise F77Error('unterminated string in ' + txt)
                if txt[j] == "'":
                    if j + 1 < len(txt) and txt[j + 1] == "'":
                        s.append("'")
                        j += 2
                        continue
                    break
                s.append(txt[j])
                j += 1
            buf.append('$%d$' % len(strings))
            strings.append(''.join(s))
            i = j + 1
            continue
        if ch not in ' \t':
            buf.append(ch.upper())
        i += 1
    return ''.join(buf), strings


# --------------------------------------------------------------------------
# Expressions
# --------------------------------------------------------------------------

_DOTOPS = ('.EQ.', '.NE.', '.LT.', '.LE.', '.GT.', '.GE.', '.AND.', '.OR.',
           '.NOT.', '.EQV.', '.NEQV.', '.TRUE.', '.FALSE.')


def tokenize(s):
    toks = []
    i = 0
    n = len(s)
    while i < n:
        ch = s[i]
        if ch == '$':
            j = s.index('$', i + 1)
            toks.append(('str', int(s[i + 1:j])))
            i = j + 1
        elif ch.isdigit() or (ch == '.' and i + 1 < n and s[i + 1].isdigit()):
            j = i
            while j < n and s[j].isdigit():
                j += 1
            is_real = False
            kind = 'f'
            if j < n and s[j] == '.' and not any(s.startswith(op, j) for op in _DOTOPS):
                is_real = True
                j += 1
                while j < n and s[j].isdigit():
                    j += 1
            if j < n and s[j] in 'ED' and (j + 1 < n) and (s[j + 1].isdigit() or
                                                           (s[j + 1] in '+-' and j + 2 < n and s[j + 2].isdigit())):
                is_real = True
                kind = 'd' if s[j] == 'D' else 'f'
                j += 1
                if s[j] in '+-':
                    j += 1
                while j < n and s[j].isdigit():
                    j += 1
            text = s[i:j]
            if is_real:
                toks.append(('real', text, kind))
            elif j + 1 < n and s[j] == '_' and s[j + 1].isalpha():
                # integer literal with a kind parameter (0_I4, 1_I8)
                k = j + 1
                while k < n and (s[k].isalnum() or s[k] == '_'):
                    k += 1
                kname = s[j + 1:k]
                if kname not in ('I4', 'I8'):
                    raise F77Error('unsupported literal kind ' + kname)
                toks.append(('int', text, kname.lower()))
                j = k
            else:
                toks.append(('int', text))
            i = j
        elif ch == '.':
            for op in _DOTOPS:
                if s.startswith(op, i):
                    toks.append(('op', op))
                    i += len(op)
                    break
            else:
                raise F77Error('bad dot token at %r' % s[i:])
        elif ch.isalpha() or ch == '_':
            j = i
            while j < n and (s[j].isalnum() or s[j] == '_'):
                j += 1
            toks.append(('name', s[i:j]))
            i = j
        elif s.startswith('**', i):
            toks.append(('op', '**'))
            i += 2
        elif s.startswith('//', i):
            toks.append(('op', '//'))
            i += 2
        elif s.startswith('::', i):
            toks.append(('op', '::'))
            i += 2
        elif ch in '+-*/(),=:':
            toks.append(('op', ch))
            i += 1
        else:
            raise F77Error('bad character %r in %r' % (ch, s))
    return toks


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else ('eof',)

    def take(self):
        tok = self.peek()
        self.i += 1
        return tok

    def expect(self, op):
        tok = self.take()
        if tok != ('op', op):
            raise F77Error('expected %s, got %r' % (op, tok))

    def at_op(self, *ops):
        tok = self.peek()
        return tok[0] == 'op' and tok[1] in ops

    def done(self):
        return self.i >= len(self.t)

    # precedence: eqv < or < and < not < rel < add < mul < pow < primary
    def expr(self):
        e = self.p_or()
        while self.at_op('.EQV.', '.NEQV.'):
            op = self.take()[1]
            e = ('bin', op, e, self.p_or())
        return e

    def p_or(self):
        e = self.p_and()
        while self.at_op('.OR.'):
            self.take()
            e = ('bin', '.OR.', e, self.p_and())
        return e

    def p_and(self):
        e = self.p_not()
        while self.at_op('.AND.'):
            self.take()
            e = ('bin', '.AND.', e, self.p_not())
        return e

    def p_not(self):
        if self.at_op('.NOT.'):
            self.take()
            return ('un', '.NOT.', self.p_not())
        return self.p_rel()

    def p_rel(self):
        e = self.p_add()
        if self.at_op('.EQ.', '.NE.', '.LT.', '.LE.', '.GT.', '.GE.'):
            op = self.take()[1]
            e = ('bin', op, e, self.p_add())
        return e

    def p_add(self):
        if self.at_op('+', '-'):
            op = self.take()[1]
            e = self.p_mul()
            if op == '-':
                e = ('un', '-', e)
        else:
            e = self.p_mul()
        while self.at_op('+', '-'):
            op = self.take()[1]
            e = ('bin', op, e, self.p_mul())
        return e

    def p_mul(self):
        e = self.p_pow()
        while self.at_op('*', '/'):
            op = self.take()[1]
            e = ('bin', op, e, self.p_pow())
        return e

    def p_pow(self):
        e = self.p_prim()
        if self.at_op('**'):
            self.take()
            if self.at_op('-', '+'):
                op = self.take()[1]
                r = self.p_pow()
                if op == '-':
                    r = ('un', '-', r)
            else:
                r = self.p_pow()
            e = ('bin', '**', e, r)
        return e

    def p_prim(self):
        tok = self.take()
        if tok[0] == 'int':
            return ('int', tok[1]) if len(tok) == 2 else ('ikind', tok[1], tok[2])
        if tok[0] == 'real':
            return ('real', tok[1], tok[2])
        if tok[0] == 'str':
            return ('str', tok[1])
        if tok == ('op', '.TRUE.'):
            return ('log', 1)
        if tok == ('op', '.FALSE.'):
            return ('log', 0)
        if tok == ('op', '('):
            e = self.expr()
            self.expect(')')
            return ('paren', e)
        if tok[0] == 'name':
            if self.at_op('('):
                self.take()
                args = []
                if not self.at_op(')'):
                    while True:
                        args.append(self.arg())
                        if self.at_op(','):
                            self.take()
                            continue
                        break
                self.expect(')')
                return ('call', tok[1], args)
            return ('name', tok[1])
        if tok[0] == 'op' and tok[1] in '+-' and False:
            pass
        raise F77Error('unexpected token %r' % (tok,))

    def arg(self):
        # keyword argument (KIND=...) or a plain expression
        if self.peek()[0] == 'name' and self.peek(1) == ('op', '='):
            name = self.take()[1]
            self.take()
            return ('kw', name, self.expr())
        return self.expr()


def parse_expr(s):
    p = Parser(tokenize(s))
    e = p.expr()
    if not p.done():
        raise F77Error('trailing tokens in expression %r' % s)
    return e


def split_top(s, sep=','):
    """Split a normalised string on `sep` at parenthesis depth 0."""
    parts = []
    depth = 0
    cur = []
    for ch in s:
        if ch == '(':
            depth += 1
        elif ch == ')':
            depth -= 1
        if ch == sep and depth == 0:
            parts.append(''.join(cur))
            cur = []
        else:
            cur.append(ch)
    parts.append(''.join(cur))
    return parts


def find_top(s, ch):
    depth = 0
    for i, c in enumerate(s):
        if c == '(':
            depth += 1
        elif c == ')':
            depth -= 1
        elif c == ch and depth == 0:
            return i
    return -1


def match_paren(s, i):
    depth = 0
    for j in range(i, len(s)):
        if s[j] == '(':
            depth += 1
        elif s[j] == ')':
            depth -= 1
            if depth == 0:
                return j
    raise F77Error('unbalanced parentheses in ' + s)


# --------------------------------------------------------------------------
# Program units
# --------------------------------------------------------------------------

class Sym:
    def __init__(self, name):
        self.name = name
        self.type = None          # 'i', 'i4', 'i8', 'l', 'd', 'f', 'c'
        self.dims = None          # list of (lb_ast, ub_ast or None for *)
        self.dummy = False
        self.param = None         # AST of a PARAMETER value
        self.external = False
        self.intrinsic = False
        self.used_as_proc = False


CTYPE = {'i': 'fint', 'l': 'fint', 'i8': 'int64_t', 'i4': 'int32_t',
         'd': 'double', 'f': 'float', 'c': 'char'}

INTRINSICS = {'ABS', 'IABS', 'DABS', 'MAX', 'MIN', 'MAX0', 'MIN0', 'DMAX1',
              'DMIN1', 'AMAX1', 'AMIN1', 'SIGN', 'ISIGN', 'DSIGN', 'MOD',
              'DBLE', 'DFLOAT', 'FLOAT', 'REAL', 'SNGL', 'INT', 'IDINT',
              'IFIX', 'NINT', 'IDNINT', 'SQRT', 'DSQRT', 'EXP', 'DEXP', 'LOG',
              'DLOG', 'HUGE', 'SELECTED_INT_KIND'}


class Unit:
    def __init__(self, kind, name, args, where):
        self.kind = kind
        self.name = name
        self.args = args
        self.where = where
        self.syms = {}
        self.implicit_none = False
        self.body = []            # executable statements (label, norm, strings, where)
        self.rettype = None
        self.stmtfuncs = {}

    def sym(self, name):
        s = self.syms.get(name)
        if s is None:
            s = self.syms[name] = Sym(name)
        return s


TYPE_RE = re.compile(r'^(DOUBLEPRECISION|INTEGER\*8|INTEGER\*4|INTEGER\((?:KIND=)?(\w+)\)|INTEGER|'
                     r'LOGICAL|REAL\*8|REAL|CHARACTER\*\(\*\)|CHARACTER\*\d+|CHARACTER)')


class Translator:
    def __init__(self, include_dirs, defines):
        self.include_dirs = include_dirs
        self.defines = defines
        self.units = []
        self.tmp = 0

    # ---------------- front end ----------------
    def load(self, path):
        # "file.f:NAME1,NAME2" translates only those routines of the file
        keep = None
        if ':' in os.path.basename(path):
            path, names = path.rsplit(':', 1)
            keep = set(n.strip().upper() for n in names.split(',') if n.strip())
        stmts = read_statements(path, self.defines, keep)
        unit = None
        for label, text, where in stmts:
            norm, strings = normalise(text)
            if unit is None:
                m = re.match(r'^(SUBROUTINE|(?:(?:DOUBLEPRECISION|INTEGER|LOGICAL|REAL)?)FUNCTION)([A-Z]\w*)(\((.*)\))?$', norm)
                if not m:
                    raise F77Error(where + ' expected SUBROUTINE/FUNCTION, got ' + norm)
                args = [a for a in (m.group(4) or '').split(',') if a]
                kind = 'sub' if m.group(1) == 'SUBROUTINE' else 'fun'
                unit = Unit(kind, m.group(2), args, where)
                if kind == 'fun':
                    pre = m.group(1)[:-len('FUNCTION')]
                    unit.rettype = {'DOUBLEPRECISION': 'd', 'INTEGER': 'i',
                                    'LOGICAL': 'l', 'REAL': 'f', '': None}[pre]
                for a in args:
                    unit.sym(a).dummy = True
                continue
            if norm == 'END' or norm in ('ENDSUBROUTINE', 'ENDFUNCTION') or \
                    norm.startswith('ENDSUBROUTINE') or norm.startswith('ENDFUNCTION'):
                self.units.append(unit)
                unit = None
                continue
            self.spec_or_exec(unit, label, norm, strings, where)
        if unit is not None:
            raise F77Error(path + ': missing END')

    def spec_or_exec(self, unit, label, norm, strings, where):
        if norm == 'IMPLICITNONE':
            unit.implicit_none = True
            return
        if norm.startswith('IMPLICIT'):
            raise F77Error(where + ' IMPLICIT other than NONE is not supported')
        if norm.startswith('INCLUDE$'):
            name = strings[int(norm[len('INCLUDE$'):-1])]
            for d in self.include_dirs:
                p = os.path.join(d, name)
                if os.path.exists(p):
                    for lab, txt, w in read_statements(p, self.defines):
                        n2, s2 = normalise(txt)
                        self.spec_or_exec(unit, lab, n2, s2, w)
                    return
            raise F77Error(where + ' include not found: ' + name)
        for kw in ('EXTERNAL', 'INTRINSIC'):
            if norm.startswith(kw) and find_top(norm, '=') < 0:
                for nm in norm[len(kw):].split(','):
                    s = unit.sym(nm)
                    if kw == 'EXTERNAL':
                        s.external = True
                    else:
                        s.intrinsic = True
                return
        if norm.startswith('SAVE') and find_top(norm, '=') < 0:
            return
        if norm.startswith('PARAMETER('):
            inner = norm[len('PARAMETER('):-1]
            for item in split_top(inner):
                k = item.index('=')
                unit.sym(item[:k]).param = parse_expr(item[k + 1:])
            return
        if norm.startswith('DIMENSION'):
            self.decl_entities(unit, None, norm[len('DIMENSION'):], where)
            return
        m = TYPE_RE.match(norm)
        if m and (find_top(norm, '=') < 0 or '::' in norm):
            spec = m.group(1)
            rest = norm[m.end():]
            if spec == 'DOUBLEPRECISION' or spec == 'REAL*8':
                ty = 'd'
            elif spec == 'REAL':
                ty = 'f'
            elif spec == 'LOGICAL':
                ty = 'l'
            elif spec.startswith('CHARACTER'):
                ty = 'c'
            elif spec == 'INTEGER':
                ty = 'i'
            elif spec == 'INTEGER*8':
                ty = 'i8'
            elif spec == 'INTEGER*4':
                ty = 'i4'
            else:
                k = m.group(2)
                kv = self.const_eval(unit, ('name', k)) if not k.isdigit() else int(k)
                ty = {8: 'i8', 4: 'i4'}[kv]
            if '::' in rest:
                attrs, ents = rest.split('::', 1)
                attrs = [a for a in attrs.split(',') if a]
                if attrs != ['PARAMETER']:
                    raise F77Error(where + ' unsupported attributes ' + rest)
                for item in split_top(ents):
                    k = item.index('=')
                    s = unit.sym(item[:k])
                    s.type = ty
                    s.param = parse_expr(item[k + 1:])
                return
            if rest.startswith(','):
                rest = rest[1:]
            self.decl_entities(unit, ty, rest, where)
            return
        if norm.startswith('DATA') and '/' in norm:
            raise F77Error(where + ' DATA statements are not supported')
        m = re.match(r'^([A-Z]\w*)\(([A-Z]\w*(?:,[A-Z]\w*)*)\)=(.*)$', norm)
        if m and not unit.body and unit.syms.get(m.group(1)) is not None \
                and unit.syms[m.group(1)].dims is None:
            # statement function: NAME(a,b) = expr
            unit.stmtfuncs[m.group(1)] = (m.group(2).split(','), parse_expr(m.group(3)))
            return
        unit.body.append((label, norm, strings, where))

    def decl_entities(self, unit, ty, rest, where):
        for ent in split_top(rest):
            if not ent:
                continue
            m = re.match(r'^([A-Z]\w*)(\*\d+|\*\(\*\))?(\((.*)\))?$', ent)
            if not m:
                raise F77Error(where + ' bad declaration entity ' + ent)
            s = unit.sym(m.group(1))
            if ty is not None:
                s.type = ty
            if m.group(3):
                dims = []
                for d in split_top(m.group(4)):
                    if d == '*':
                        dims.append((('int', '1'), None))
                    elif find_top(d, ':') >= 0:
                        k = find_top(d, ':')
                        ub = d[k + 1:]
                        dims.append((parse_expr(d[:k]), None if ub == '*' else parse_expr(ub)))
                    else:
                        dims.append((('int', '1'), parse_expr(d)))
                s.dims = dims

    # ---------------- helpers ----------------
    def const_eval(self, unit, e):
        k = e[0]
        if k in ('int', 'ikind'):
            return int(e[1])
        if k == 'paren':
            return self.const_eval(unit, e[1])
        if k == 'name':
            s = unit.syms.get(e[1])
            if s is None or s.param is None:
                raise F77Error('not a constant: ' + e[1])
            return self.const_eval(unit, s.param)
        if k == 'un' and e[1] == '-':
            return -self.const_eval(unit, e[2])
        if k == 'bin':
            a = self.const_eval(unit, e[2])
            b = self.const_eval(unit, e[3])
            if e[1] == '+':
                return a + b
            if e[1] == '-':
                return a - b
            if e[1] == '*':
                return a * b
            if e[1] == '/':
                return int(a / b)
            if e[1] == '**':
                return a ** b
        if k == 'call' and e[1] == 'SELECTED_INT_KIND':
            r = self.const_eval(unit, e[2][0])
            return 4 if r <= 9 else 8
        raise F77Error('cannot fold constant %r' % (e,))

    def type_of_name(self, unit, name):
        s = unit.syms.get(name)
        if s is not None and s.type is not None:
            return s.type
        if unit.implicit_none and not (s is not None and s.param is not None):
            raise F77Error('%s: undeclared name %s under IMPLICIT NONE' % (unit.name, name))
        if s is not None and s.param is not None:
            return self.expr_type(unit, s.param)
        return 'i' if name[0] in 'IJKLMN' else 'f'

    def expr_type(self, unit, e):
        k = e[0]
        if k == 'int':
            return 'i'
        if k == 'ikind':
            return e[2]
        if k == 'real':
            return 'd' if e[2] == 'd' else 'f'
        if k == 'log':
            return 'l'
        if k == 'str':
            return 'c'
        if k == 'paren':
            return self.expr_type(unit, e[1])
        if k == 'name':
            return self.type_of_name(unit, e[1])
        if k == 'un':
            return 'l' if e[1] == '.NOT.' else self.expr_type(unit, e[2])
        if k == 'bin':
            if e[1] in ('.EQ.', '.NE.', '.LT.', '.LE.', '.GT.', '.GE.', '.AND.',
                        '.OR.', '.EQV.', '.NEQV.'):
                return 'l'
            return promote(self.expr_type(unit, e[2]), self.expr_type(unit, e[3]))
        if k == 'call':
            name = e[1]
            s = unit.syms.get(name)
            if s is not None and s.dims is not None:
                return self.type_of_name(unit, name)
            if name in INTRINSICS and not (s is not None and s.external):
                return self.intrinsic_type(unit, name, e[2])
            if s is not None and s.type is not None:
                return s.type
            return 'i' if name[0] in 'IJKLMN' else 'f'
        raise F77Error('type of %r' % (e,))

    def intrinsic_type(self, unit, name, args):
        ts = [self.expr_type(unit, a) for a in args if a[0] != 'kw']
        if name == 'SELECTED_INT_KIND':
            return 'i'
        if name in ('ABS', 'MAX', 'MIN', 'SIGN', 'MOD'):
            t = ts[0]
            for x in ts[1:]:
                t = promote(t, x)
            return t
        if name == 'INT' and len(args) == 2:
            a1 = args[1][2] if args[1][0] == 'kw' else args[1]
            return {8: 'i8', 4: 'i4'}[self.const_eval(unit, a1)]
        if name in ('IABS', 'MAX0', 'MIN0', 'ISIGN', 'INT', 'IDINT', 'IFIX', 'NINT', 'IDNINT',
                    'SELECTED_INT_KIND'):
            return 'i'
        if name in ('DABS', 'DMAX1', 'DMIN1', 'DSIGN', 'DBLE', 'DFLOAT', 'DSQRT', 'DEXP', 'DLOG'):
            return 'd'
        if name in ('FLOAT', 'REAL', 'SNGL', 'AMAX1', 'AMIN1'):
            return 'f'
        if name in ('SQRT', 'EXP', 'LOG'):
            return ts[0]
        if name == 'HUGE':
            return ts[0]
        raise F77Error('intrinsic ' + name)

    # ---------------- C emission of expressions ----------------
    def c_name(self, unit, name):
        s = unit.syms[name]
        if s.dummy and s.dims is None:
            return '(*%s)' % name
        return name

    def c_index(self, unit, name, subs):
        s = unit.syms[name]
        dims = s.dims
        if len(subs) != len(dims):
            raise F77Error('%s: rank mismatch for %s' % (unit.name, name))
        terms = []
        mult = None
        for k, (sub, (lb, ub)) in enumerate(zip(subs, dims)):
            lbc = self.c_expr(unit, lb)
            term = '((%s)-(%s))' % (self.c_expr(unit, sub), lbc)
            if mult:
                term = '%s*%s' % (term, mult)
            terms.append(term)
            if k + 1 < len(dims):
                ext = '_x_%s_%d' % (name, k)
                mult = ext if mult is None else '%s*%s' % (mult, ext)
        return '%s[%s]' % (name, '+'.join(terms))

    def c_expr(self, unit, e):
        k = e[0]
        if k == 'int':
            return '((fint)%s)' % e[1]
        if k == 'ikind':
            return '((%s)%s)' % ('int32_t' if e[2] == 'i4' else 'int64_t', e[1])
        if k == 'real':
            txt = e[1].replace('D', 'e').replace('E', 'e')
            if '.' not in txt and 'e' not in txt:
                txt += '.'
            if txt.endswith('.') or txt.startswith('.'):
                txt = txt.replace('.e', '.0e')
                if txt.endswith('.'):
                    txt += '0'
                if txt.startswith('.'):
                    txt = '0' + txt
            return '(%s)' % txt if e[2] == 'd' else '(%sf)' % txt
        if k == 'log':
            return '((fint)%d)' % e[1]
        if k == 'str':
            return '"%s"' % self.strings[e[1]].replace('\\', '\\\\').replace('"', '\\"')
        if k == 'paren':
            return '(%s)' % self.c_expr(unit, e[1])
        if k == 'name':
            s = unit.syms.get(e[1])
            if s is None:
                unit.sym(e[1])
                s = unit.syms[e[1]]
            if s.param is not None:
                t = self.type_of_name(unit, e[1])
                return '((%s)(%s))' % (CTYPE[t], self.c_expr(unit, s.param))
            return self.c_name(unit, e[1])
        if k == 'un':
            if e[1] == '.NOT.':
                return '(!%s)' % self.c_expr(unit, e[2])
            return '(-%s)' % self.c_expr(unit, e[2])
        if k == 'bin':
            op = e[1]
            a = self.c_expr(unit, e[2])
            b = self.c_expr(unit, e[3])
            cop = {'.EQ.': '==', '.NE.': '!=', '.LT.': '<', '.LE.': '<=', '.GT.': '>',
                   '.GE.': '>=', '.AND.': '&&', '.OR.': '||', '+': '+', '-': '-', '*': '*',
                   '/': '/'}.get(op)
            if cop:
                return '(%s %s %s)' % (a, cop, b)
            if op == '.EQV.':
                return '((!%s) == (!%s))' % (a, b)
            if op == '.NEQV.':
                return '((!%s) != (!%s))' % (a, b)
            if op == '**':
                ta = self.expr_type(unit, e[2])
                tb = self.expr_type(unit, e[3])
                if ta in ('i', 'i4', 'i8') and tb in ('i', 'i4', 'i8'):
                    return 'f77_ipow(%s, %s)' % (a, b)
                if tb in ('i', 'i4', 'i8'):
                    fn = '__builtin_powi' if ta == 'd' else '__builtin_powif'
                    return '%s(%s, (int)(%s))' % (fn, a, b)
                return 'pow(%s, %s)' % (a, b)
            raise F77Error('operator ' + op)
        if k == 'call':
            name = e[1]
            args = e[2]
            s = unit.syms.get(name)
            if s is not None and s.dims is not None:
                return self.c_index(unit, name, args)
            if name in unit.stmtfuncs:
                return '((%s)%s)' % (CTYPE[self.type_of_name(unit, name)],
                                     self.c_expr(unit, self.expand_sf(unit, name, args)))
            if name in INTRINSICS and not (s is not None and s.external):
                return self.c_intrinsic(unit, name, args)
            # user function
            return '%s(%s)' % (self.c_callee(unit, name), ', '.join(self.c_arg(unit, a) for a in args))
        raise F77Error('expression %r' % (e,))

    def expand_sf(self, unit, name, args):
        params, body = unit.stmtfuncs[name]
        env = dict(zip(params, [('paren', a) for a in args]))

        def sub(e):
            if e[0] == 'name' and e[1] in env:
                return env[e[1]]
            if e[0] == 'paren':
                return ('paren', sub(e[1]))
            if e[0] == 'un':
                return ('un', e[1], sub(e[2]))
            if e[0] == 'bin':
                return ('bin', e[1], sub(e[2]), sub(e[3]))
            if e[0] == 'call':
                return ('call', e[1], [sub(x) for x in e[2]])
            return e
        return ('paren', sub(body))

    def c_intrinsic(self, unit, name, args):
        cs = [self.c_expr(unit, a) for a in args]
        t = self.intrinsic_type(unit, name, args)
        isint = t in ('i', 'i4', 'i8', 'l')
        if name in ('ABS', 'IABS', 'DABS'):
            if isint:
                return 'f77_iabs(%s)' % cs[0]
            return ('fabs(%s)' if t == 'd' else 'fabsf(%s)') % cs[0]
        if name in ('MAX', 'MIN', 'MAX0', 'MIN0', 'DMAX1', 'DMIN1', 'AMAX1', 'AMIN1'):
            f = 'max' if 'MAX' in name else 'min'
            fn = ('f77_i' if isint else 'f77_d') + f
            acc = cs[0]
            for c in cs[1:]:
                acc = '%s(%s, %s)' % (fn, acc, c)
            return acc
        if name in ('SIGN', 'ISIGN', 'DSIGN'):
            if isint:
                return 'f77_isign(%s, %s)' % (cs[0], cs[1])
            return 'copysign(fabs(%s), %s)' % (cs[0], cs[1])
        if name == 'MOD':
            if isint:
                return '((%s) %% (%s))' % (cs[0], cs[1])
            return 'fmod(%s, %s)' % (cs[0], cs[1])
        if name in ('DBLE', 'DFLOAT'):
            return '((double)(%s))' % cs[0]
        if name in ('FLOAT', 'REAL', 'SNGL'):
            return '((float)(%s))' % cs[0]
        if name in ('INT', 'IDINT', 'IFIX'):
            if len(args) == 2:
                kv = self.const_eval(unit, args[1][2] if args[1][0] == 'kw' else args[1])
                return '((%s)(%s))' % ({8: 'int64_t', 4: 'int32_t'}[kv], cs[0])
            return '((fint)(%s))' % cs[0]
        if name == 'SELECTED_INT_KIND':
            return '((fint)%d)' % self.const_eval(unit, ('call', name, args))
        if name in ('NINT', 'IDNINT'):
            return '((fint)llround(%s))' % cs[0]
        if name in ('SQRT', 'DSQRT'):
            return ('sqrt(%s)' if t == 'd' else 'sqrtf(%s)') % cs[0]
        if name in ('EXP', 'DEXP'):
            return 'exp(%s)' % cs[0]
        if name in ('LOG', 'DLOG'):
            return 'log(%s)' % cs[0]
        if name == 'HUGE':
            return 'FINT_MAX' if isint else 'DBL_MAX'
        raise F77Error('intrinsic ' + name)

    def c_callee(self, unit, name):
        s = unit.syms.get(name)
        if s is not None and s.dummy:
            s.used_as_proc = True
            return '((void (*)())%s)' % name
        return name.lower() + '_'

    def c_arg(self, unit, a):
        k = a[0]
        if k == 'name':
            s = unit.syms.get(a[0 + 1])
            name = a[1]
            if s is None:
                s = unit.sym(name)
            if s.param is not None:
                t = self.type_of_name(unit, name)
                return '(void *)&(%s){%s}' % (CTYPE[t], self.c_expr(unit, a))
            if s.dummy:
                return '(void *)%s' % name
            if s.external or (s.type is None and not s.dims and name.lower() + '_' in self.routines):
                return '(void *)%s_' % name.lower()
            if s.dims is not None:
                return '(void *)%s' % name
            return '(void *)&%s' % name
        if k == 'call':
            s = unit.syms.get(a[1])
            if s is not None and s.dims is not None:
                return '(void *)&%s' % self.c_index(unit, a[1], a[2])
        if k == 'str':
            return '(void *)%s' % self.c_expr(unit, a)
        t = self.expr_type(unit, a)
        return '(void *)&(%s){%s}' % (CTYPE[t], self.c_expr(unit, a))

    # ---------------- statements ----------------
    def emit_unit(self, unit):
        out = []
        self.strings = None
        params = []
        for a in unit.args:
            s = unit.syms[a]
            if s.external or self._is_proc_dummy(unit, a):
                params.append('void *%s' % a)
            else:
                t = s.type or ('i' if a[0] in 'IJKLMN' else 'f')
                if s.type is None:
                    if unit.implicit_none:
                        raise F77Error('%s: undeclared dummy %s' % (unit.name, a))
                    s.type = t
                params.append('%s *%s' % (CTYPE[t], a))
        rt = 'void'
        if unit.kind == 'fun':
            rt = CTYPE[unit.rettype or self.type_of_name(unit, unit.name)]
        body = []
        self.label_stack = []
        self.gen_body(unit, body)
        # declarations (after the body so implicit locals are known)
        decl = []
        for a in unit.args:
            s = unit.syms[a]
            if s.dims and len(s.dims) > 1:
                for kk, (lb, ub) in enumerate(s.dims[:-1]):
                    decl.append('    const fint _x_%s_%d = (%s) - (%s) + 1;' % (
                        a, kk, self.c_expr(unit, ub), self.c_expr(unit, lb)))
        for name, s in sorted(unit.syms.items()):
            if s.dummy or s.param is not None or s.external or s.intrinsic:
                continue
            if name in INTRINSICS and s.type is None and s.dims is None:
                continue
            if name.lower() + '_' in self.routines and s.type is None:
                continue
            if unit.kind == 'fun' and name == unit.name:
                continue
            if name in unit.stmtfuncs:
                continue
            t = s.type or self.type_of_name(unit, name)
            if s.dims is not None:
                size = 1
                for kk, (lb, ub) in enumerate(s.dims):
                    ext = self.const_eval(unit, ub) - self.const_eval(unit, lb) + 1
                    size *= ext
                    if kk + 1 < len(s.dims):
                        decl.append('    const fint _x_%s_%d = %d;' % (name, kk, ext))
                decl.append('    %s %s[%d] = {0};' % (CTYPE[t], name, size))
            else:
                decl.append('    %s %s = 0;' % (CTYPE[t], name))
        if unit.kind == 'fun':
            decl.append('    %s %s = 0;' % (rt, unit.name))
        out.append('/* %s */' % unit.where)
        out.append('%s %s_(%s)\n{' % (rt, unit.name.lower(), ', '.join(params) or 'void'))
        out.extend(decl)
        out.extend(body)
        if unit.kind == 'fun':
            out.append('    return %s;' % unit.name)
        out.append('}\n')
        return '\n'.join(out)

    def _is_proc_dummy(self, unit, name):
        # a dummy that is CALLed (or passed where a routine is expected)
        for label, norm, strings, where in unit.body:
            m = re.match(r'^(?:IF\(.*\))?CALL([A-Z]\w*)', norm)
            if m and m.group(1) == name:
                return True
        return False

    def gen_body(self, unit, out):
        stack = []                 # ('do', label) | ('if',)
        self.tmp = 0
        for label, norm, strings, where in unit.body:
            self.strings = strings
            try:
                self.gen_stmt(unit, label, norm, where, stack, out)
            except F77Error as exc:
                raise F77Error('%s: %s (%s)' % (where, exc, norm))
        if stack:
            raise F77Error('%s: unclosed blocks %r' % (unit.name, stack))

    def gen_stmt(self, unit, label, norm, where, stack, out):
        ind = '    ' * (len(stack) + 1)
        lab = 'L%s: ;' % label if label else None
        if norm in ('ENDDO',):
            if lab:
                out.append(ind + lab)
            if not stack or stack[-1][0] != 'do':
                raise F77Error('END DO without DO')
            stack.pop()
            out.append('    ' * (len(stack) + 1) + '}}')
            return
        if norm == 'ENDIF':
            if not stack or stack[-1][0] != 'if':
                raise F77Error('END IF without IF')
            stack.pop()
            out.append('    ' * (len(stack) + 1) + '}')
            if lab:
                out.append('    ' * (len(stack) + 1) + lab)
            return
        if norm == 'ELSE':
            out.append('    ' * len(stack) + '} else {')
            return
        m = re.match(r'^ELSEIF(\(.*\))THEN$', norm)
        if m:
            cond = parse_expr(m.group(1))
            out.append('    ' * len(stack) + '} else if (%s) {' % self.c_expr(unit, cond))
            return
        if lab:
            out.append(ind + lab)
        if norm.startswith('IF('):
            j = match_paren(norm, 2)
            cond = parse_expr(norm[2:j + 1])
            rest = norm[j + 1:]
            if rest == 'THEN':
                out.append(ind + 'if (%s) {' % self.c_expr(unit, cond))
                stack.append(('if',))
                return
            m = re.match(r'^(\d+),(\d+),(\d+)$', rest)
            if m:
                t = self.expr_type(unit, cond)
                out.append(ind + '{ %s _a = %s; if (_a < 0) goto L%s; else if (_a == 0) goto L%s; else goto L%s; }'
                           % (CTYPE[t], self.c_expr(unit, cond), m.group(1), m.group(2), m.group(3)))
                self._close_do(label, stack, out)
                return
            sub = []
            self.simple_stmt(unit, rest, sub)
            out.append(ind + 'if (%s) { %s }' % (self.c_expr(unit, cond), ' '.join(sub)))
            self._close_do(label, stack, out)
            return
        m = re.match(r'^DO(\d+),?([A-Z]\w*)=(.*)$', norm)
        m2 = re.match(r'^DO([A-Z]\w*)=(.*)$', norm)
        if m and len(split_top(m.group(3))) >= 2:
            self.gen_do(unit, m.group(2), m.group(3), m.group(1), ind, stack, out)
            return
        if m2 and len(split_top(m2.group(2))) >= 2:
            self.gen_do(unit, m2.group(1), m2.group(2), None, ind, stack, out)
            return
        sub = []
        self.simple_stmt(unit, norm, sub)
        for s in sub:
            out.append(ind + s)
        self._close_do(label, stack, out)

    def _close_do(self, label, stack, out):
        if not label:
            return
        while stack and stack[-1] == ('do', label):
            stack.pop()
            out.append('    ' * (len(stack) + 1) + '}}')

    def gen_do(self, unit, var, ctl, label, ind, stack, out):
        parts = [parse_expr(p) for p in split_top(ctl)]
        v = self.c_expr(unit, ('name', var))
        vt = CTYPE[self.type_of_name(unit, var)]
        self.tmp += 1
        n = self.tmp
        lb = self.c_expr(unit, parts[0])
        ub = self.c_expr(unit, parts[1])
        if len(parts) == 2:
            out.append(ind + '{ const %s _u%d = %s; for (%s = %s; %s <= _u%d; %s++) {'
                       % (vt, n, ub, v, lb, v, n, v))
        else:
            st = self.c_expr(unit, parts[2])
            out.append(ind + '{ const %s _u%d = %s, _s%d = %s; for (%s = %s; _s%d > 0 ? %s <= _u%d : %s >= _u%d; %s += _s%d) {'
                       % (vt, n, ub, n, st, v, lb, n, v, n, v, n, v, n))
        stack.append(('do', label))

    def simple_stmt(self, unit, norm, out):
        if norm == 'CONTINUE':
            out.append(';')
            return
        if norm == 'RETURN':
            out.append('return%s;' % ((' ' + unit.name) if unit.kind == 'fun' else ''))
            return
        if norm.startswith('STOP'):
            out.append('abort();')
            return
        m = re.match(r'^GOTO(\d+)$', norm)
        if m:
            out.append('goto L%s;' % m.group(1))
            return
        m = re.match(r'^GOTO\(([\d,]+)\),?(.*)$', norm)
        if m:
            labels = m.group(1).split(',')
            sel = self.c_expr(unit, parse_expr(m.group(2)))
            cases = ' '.join('case %d: goto L%s;' % (i + 1, l) for i, l in enumerate(labels))
            out.append('switch ((fint)(%s)) { %s default: break; }' % (sel, cases))
            return
        if norm.startswith('WRITE(') or norm.startswith('PRINT') or norm.startswith('FORMAT(') \
                or norm.startswith('READ('):
            out.append(';')
            return
        m = re.match(r'^CALL([A-Z]\w*)(\((.*)\))?$', norm)
        if m:
            name = m.group(1)
            args = []
            if m.group(2) and m.group(3):
                p = Parser(tokenize(m.group(3)))
                while True:
                    args.append(p.expr())
                    if p.at_op(','):
                        p.take()
                        continue
                    break
                if not p.done():
                    raise F77Error('bad CALL arguments')
            out.append('%s(%s);' % (self.c_callee(unit, name), ', '.join(self.c_arg(unit, a) for a in args)))
            return
        k = find_top(norm, '=')
        if k > 0:
            lhs = parse_expr(norm[:k])
            rhs = parse_expr(norm[k + 1:])
            if lhs[0] == 'name' and unit.kind == 'fun' and lhs[1] == unit.name:
                out.append('%s = %s;' % (unit.name, self.c_expr(unit, rhs)))
                return
            out.append('%s = %s;' % (self.c_expr(unit, lhs), self.c_expr(unit, rhs)))
            return
        raise F77Error('unsupported statement')

    def translate(self, paths):
        for p in paths:
            self.load(p)
        self.routines = set(u.name.lower() + '_' for u in self.units)
        parts = [PRELUDE]
        for u in self.units:
            rt = 'void'
            if u.kind == 'fun':
                rt = CTYPE[u.rettype or 'f']
            parts.append('%s %s_();' % (rt, u.name.lower()))
        # typed EXTERNAL functions defined outside this translation (BLAS,
        # other libraries): their return type must be declared
        ext = {}
        for u in self.units:
            for sym in u.syms.values():
                nm = sym.name.lower() + '_'
                if sym.external and sym.type is not None and not sym.dummy and nm not in self.routines:
                    ext[nm] = CTYPE[sym.type]
        for nm in sorted(ext):
            parts.append('%s %s();' % (ext[nm], nm))
        parts.append('')
        for u in self.units:
            parts.append(self.emit_unit(u))
        return '\n'.join(parts)


def promote(a, b):
    order = {'l': 0, 'i4': 1, 'i': 2, 'i8': 3, 'f': 4, 'd': 5, 'c': -1}
    return a if order[a] >= order[b] else b


PRELUDE = r'''/* Machine translation of the SPR Fortran sources (oracle build output,
 * never committed).  Generated by oracle/f77c.py. */
#include <stdint.h>
#include <stdlib.h>
#include <math.h>
#include <float.h>
#ifndef FINT
#define FINT int64_t
#endif
typedef FINT fint;
#define FINT_MAX ((fint)((((uint64_t)1) << (8 * sizeof(fint) - 1)) - 1))
static inline fint f77_iabs(fint a) { return a < 0 ? -a : a; }
static inline fint f77_imax(fint a, fint b) { return a > b ? a : b; }
static inline fint f77_imin(fint a, fint b) { return a < b ? a : b; }
static inline double f77_dmax(double a, double b) { return a > b ? a : b; }
static inline double f77_dmin(double a, double b) { return a < b ? a : b; }
static inline fint f77_isign(fint a, fint b) { return b >= 0 ? f77_iabs(a) : -f77_iabs(a); }
static inline fint f77_ipow(fint b, fint e) {
    fint r = 1;
    if (e < 0) return (b == 1) ? 1 : (b == -1 ? ((e & 1) ? -1 : 1) : 0);
    while (e) { if (e & 1) r *= b; b *= b; e >>= 1; }
    return r;
}
'''


def main(argv):
    import argparse
    ap = argparse.ArgumentParser(description=__doc__.split('\n')[0])
    ap.add_argument('-o', '--output', required=True)
    ap.add_argument('-I', dest='incs', action='append', default=[])
    ap.add_argument('sources', nargs='+')
    a = ap.parse_args(argv)
    incs = a.incs or sorted(set(os.path.dirname(os.path.abspath(s)) for s in a.sources))
    tr = Translator(incs, defines={})
    code = tr.translate(a.sources)
    os.makedirs(os.path.dirname(os.path.abspath(a.output)), exist_ok=True)
    with open(a.output, 'w') as fh:
        fh.write(code)


if __name__ == '__main__':
    main(sys.argv[1:])
