"""Run the reference's own Python 2 modules, unmodified on disk, in this
Python 3, to generate golden fixtures.  TEST INFRASTRUCTURE ONLY: used by
tests/golden/make_golden_py_ref.py (and by CPU tests that re-check the
fixtures when the reference checkout is present); nothing in the package,
bench.py or a GPU test imports it.

freifeld/cpabDiffeo is Python 2 and imports the author's external package
`of` (absent).  A module is loaded by reading its source from the checkout
and applying, in memory, only mechanical changes that keep Python 2's
meaning:

  1. print statements become print() calls (token-level rewrite);
  2. every `/` and `/=` becomes __py2div__(a, b): floor division when both
     operands are integers (Python ints, numpy integer scalars or integer
     arrays), true division otherwise -- Python 2's classic division;
  3. zip, map, filter and range return lists, xrange is range (the
     Python 2 builtins);
  4. implicit relative imports (`from _PAT import PAT`) load the sibling
     file; `cpab.<pkg>` packages are resolved lazily from the `from X import
     Y` lines of their __init__.py, so importing one name does not import
     the whole package (whose CUDA launcher needs pycuda); `of`, `of.utils`
     and `pylab` are stubs (ipshell raises; the exception classes exist);
  5. numpy names removed in numpy 2 (np.int, np.float, np.bool) are aliased
     to the builtins they were aliases of.

Nothing else of the source changes; the module's own functions run.
"""
from __future__ import annotations

import ast
import builtins
import io
import os
import sys
import tokenize
import types
from pathlib import Path

import numpy as np


def reference_root() -> Path | None:
    """The cpabDiffeo checkout: $CPAB_REF_ROOT, else the build container's mount."""
    for cand in (os.environ.get("CPAB_REF_ROOT"), "/root/reference"):
        if cand and (Path(cand) / "cpab").is_dir():
            return Path(cand)
    return None


# ----------------------------------------------------------------------------- source rewrites


def fix_print_statements(src: str) -> str:
    """Turn Python 2 print statements into calls, token by token."""
    toks = list(tokenize.generate_tokens(io.StringIO(src).readline))
    starts = [0]
    for ln in src.splitlines(keepends=True):
        starts.append(starts[-1] + len(ln))

    def off(pos):
        return starts[pos[0] - 1] + pos[1]

    edits = []  # (start, end, replacement), non-overlapping
    stmt_start = True
    i = 0
    while i < len(toks):
        t = toks[i]
        if t.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT):
            stmt_start = True
            i += 1
            continue
        if t.type in (tokenize.NL, tokenize.COMMENT):
            i += 1
            continue
        if stmt_start and t.type == tokenize.NAME and t.string == "print":
            # the statement's significant tokens after `print`
            body, depth, j = [], 0, i + 1
            while j < len(toks):
                u = toks[j]
                if depth == 0 and (u.type in (tokenize.NEWLINE, tokenize.ENDMARKER) or
                                   (u.type == tokenize.OP and u.string == ";")):
                    break
                if u.type == tokenize.OP and u.string in "([{":
                    depth += 1
                elif u.type == tokenize.OP and u.string in ")]}":
                    depth -= 1
                if u.type not in (tokenize.NL, tokenize.COMMENT):
                    body.append(j)
                j += 1
            if not body:
                edits.append((off(t.end), off(t.end), "()"))
            elif not (toks[body[0]].string == "(" and _close_of(toks, body[0]) == body[-1]):
                if toks[body[0]].string == ">>":
                    raise NotImplementedError("print >> redirection")
                last = toks[body[-1]]
                edits.append((off(t.end), off(toks[body[0]].start), "("))
                if last.type == tokenize.OP and last.string == ",":
                    edits.append((off(last.start), off(last.end), ", end=' ')"))
                else:
                    edits.append((off(last.end), off(last.end), ")"))
            stmt_start = False
            i = j
            continue
        # a one-line compound statement: `if x: print y`
        stmt_start = (t.type == tokenize.OP and t.string == ":" and _ends_header(toks, i))
        i += 1
    out = src
    for s0, s1, rep in sorted(edits, key=lambda e: -e[0]):
        out = out[:s0] + rep + out[s1:]
    return out


def _close_of(toks, i):
    """Index of the bracket closing the one at toks[i]."""
    depth = 0
    for j in range(i, len(toks)):
        u = toks[j]
        if u.type == tokenize.OP and u.string in "([{":
            depth += 1
        elif u.type == tokenize.OP and u.string in ")]}":
            depth -= 1
            if depth == 0:
                return j
    return -1


def _ends_header(toks, i):
    """A ':' at bracket depth 0 that ends a compound-statement header with
    more of the statement on the same line (`if x: print y`)."""
    depth = 0
    first = None
    for k in range(i - 1, -1, -1):
        u = toks[k]
        if u.type in (tokenize.NEWLINE, tokenize.INDENT, tokenize.DEDENT, tokenize.NL) and depth == 0:
            break
        if u.type == tokenize.OP and u.string in ")]}":
            depth += 1
        elif u.type == tokenize.OP and u.string in "([{":
            depth -= 1
            if depth < 0:
                return False
        first = u
    if depth != 0 or first is None or first.type != tokenize.NAME:
        return False
    if first.string not in ("if", "elif", "else", "for", "while", "try", "except", "finally", "with", "def",
                            "class"):
        return False
    return i + 1 < len(toks) and toks[i + 1].type not in (tokenize.NEWLINE, tokenize.NL, tokenize.COMMENT)


class _ClassicDivision(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            return ast.copy_location(ast.Call(ast.Name("__py2div__", ast.Load()), [node.left, node.right], []), node)
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            tgt_load = _as_load(node.target)
            call = ast.Call(ast.Name("__py2div__", ast.Load()), [tgt_load, node.value], [])
            return ast.copy_location(ast.Assign([node.target], call), node)
        return node


def _as_load(t):
    t2 = ast.parse(ast.unparse(t), mode="eval").body
    return t2


def _is_int(x) -> bool:
    if isinstance(x, bool):
        return True
    if isinstance(x, (int, np.integer)):
        return True
    if isinstance(x, np.ndarray):
        return np.issubdtype(x.dtype, np.integer) or x.dtype == np.bool_
    return False


def py2div(a, b):
    if _is_int(a) and _is_int(b):
        return a // b
    return a / b


# ----------------------------------------------------------------------------- stubs and imports


class _Ipshell(Exception):
    pass


def _make_of_stubs():
    of = types.ModuleType("of")
    utils = types.ModuleType("of.utils")

    def ipshell(*a, **k):
        raise _Ipshell(f"the reference called ipshell{a!r}")

    class ObsoleteError(Exception):
        pass

    class FileDoesNotExistError(Exception):
        pass

    class Bunch(dict):
        def __getattr__(self, k):
            try:
                return self[k]
            except KeyError as ex:
                raise AttributeError(k) from ex

        def __setattr__(self, k, v):
            self[k] = v

    utils.ipshell = ipshell
    utils.Bunch = Bunch
    utils.ObsoleteError = ObsoleteError
    utils.FileDoesNotExistError = FileDoesNotExistError
    utils.np = np
    utils.__all__ = ["ipshell", "Bunch", "ObsoleteError", "FileDoesNotExistError", "np"]
    of.utils = utils
    pylab = types.ModuleType("pylab")
    pylab.plt = types.SimpleNamespace()
    return {"of": of, "of.utils": utils, "pylab": pylab}


class Py2Loader:
    """Loads reference modules from a checkout with the rewrites above."""

    def __init__(self, root: Path | None = None):
        self.root = Path(root) if root else reference_root()
        if self.root is None:
            raise FileNotFoundError("no cpabDiffeo checkout (set CPAB_REF_ROOT)")
        self.modules: dict[str, types.ModuleType] = {}
        self.stubs = _make_of_stubs()
        for name in ("int", "float", "bool", "object"):
            if name not in np.__dict__:
                setattr(np, name, getattr(builtins, name))
        self._builtins = dict(builtins.__dict__)
        self._builtins.update({
            "__import__": self._import,
            "__py2div__": py2div,
            "zip": lambda *a: list(builtins.zip(*a)),
            "map": lambda f, *a: list(builtins.map(f, *a)),
            "filter": lambda f, a: list(builtins.filter(f, a)),
            "range": lambda *a: list(builtins.range(*a)),
            "xrange": builtins.range,
        })

    # a module by path relative to the checkout, e.g. "cpab/cpa1d/calcs/ClosedFormInt.py"
    def load(self, rel: str) -> types.ModuleType:
        path = (self.root / rel).resolve()
        key = str(path)
        if key in self.modules:
            return self.modules[key]
        src = path.read_text()
        src = fix_print_statements(src)
        tree = _ClassicDivision().visit(ast.parse(src, filename=str(path)))
        ast.fix_missing_locations(tree)
        code = compile(tree, str(path), "exec")
        mod = types.ModuleType(self._dotted(path))
        mod.__file__ = str(path)
        mod.__dict__["__builtins__"] = self._builtins
        self.modules[key] = mod
        exec(code, mod.__dict__)
        return mod

    def _dotted(self, path: Path) -> str:
        rel = path.relative_to(self.root).with_suffix("")
        return "refpy2." + ".".join(rel.parts)

    def _package(self, pkg_dir: Path) -> types.ModuleType:
        key = str(pkg_dir.resolve())
        if key in self.modules:
            return self.modules[key]
        init = pkg_dir / "__init__.py"
        names: dict[str, tuple[str, str]] = {}
        if init.exists():
            for node in ast.walk(ast.parse(fix_print_statements(init.read_text()))):
                if isinstance(node, ast.ImportFrom) and node.level == 0 and node.module:
                    for al in node.names:
                        names[al.asname or al.name] = (node.module, al.name)
        loader = self

        class LazyPackage(types.ModuleType):
            def __getattr__(self, attr):
                sub = pkg_dir / attr
                if attr in names:
                    modname, orig = names[attr]
                    if orig == "*":
                        raise AttributeError(attr)
                    m = loader._resolve(modname, pkg_dir)
                    val = getattr(m, orig)
                elif (sub.with_suffix(".py")).exists():
                    val = loader.load(str(sub.with_suffix(".py").relative_to(loader.root)))
                elif sub.is_dir():
                    val = loader._package(sub)
                else:
                    raise AttributeError(f"{pkg_dir.name}.{attr}")
                setattr(self, attr, val)
                return val

        mod = LazyPackage(self._dotted(pkg_dir / "__init__"))
        mod.__path__ = [str(pkg_dir)]
        self.modules[key] = mod
        return mod

    def _resolve(self, name: str, here: Path):
        """Module `name` as imported from a file in directory `here`."""
        if name in self.stubs:
            return self.stubs[name]
        parts = name.split(".")
        if parts[0] == "cpab":
            base = self.root
        else:
            base = here
            if not ((here / parts[0]).with_suffix(".py").exists() or (here / parts[0]).is_dir()):
                return None
        p = base
        mod = None
        for k, part in enumerate(parts):
            p = p / part
            if p.with_suffix(".py").exists():
                mod = self.load(str(p.with_suffix(".py").relative_to(self.root)))
            elif p.is_dir():
                mod = self._package(p)
            else:
                raise ImportError(f"{name} from {here}")
        return mod

    def _import(self, name, globals=None, locals=None, fromlist=(), level=0):
        here = Path(globals["__file__"]).parent if globals and "__file__" in globals else None
        if name in self.stubs:
            return self.stubs[name] if fromlist else self.stubs[name.split(".")[0]]
        if level == 0 and here is not None:
            mod = self._resolve(name, here)
            if mod is not None:
                if fromlist:
                    return mod
                return self._resolve(name.split(".")[0], here)
        return builtins.__import__(name, globals, locals, fromlist, level)
