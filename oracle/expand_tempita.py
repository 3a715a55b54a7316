"""ORACLE build step: expand one of the reference's Tempita templates
(src/*.c.in, src/*.h.in) into plain C under oracle/_ref/gen/.

The reference's own build does the same with the `tempita` package
(wscript:416-433).  That package is not installed; Cython ships a copy as
Cython.Tempita, whose pure-Python source (Cython/Tempita/_tempita.py) is used
here.  Under Python 3.12 its ``{{def f(a, b)}}`` signature parser drops every
argument, because tokenize now emits a NEWLINE token before ENDMARKER; the
copy loaded below sees a tokenize whose token stream omits NEWLINE/NL, which
restores the parser's intended behaviour.  The templates also rely on the
Python 2 list-returning zip(); the expansion namespace provides one.  The output is a build product of
the reference's sources and stays git-ignored.
"""
import importlib.util
import os
import sys
import tokenize as _tokenize
import types

import Cython.Tempita


class _TokenizeWithoutNewlines(types.ModuleType):
    def __init__(self):
        super().__init__("tokenize_without_newlines")
        self.__dict__.update({k: getattr(_tokenize, k) for k in dir(_tokenize)
                              if not k.startswith("__")})
        self.generate_tokens = _generate_tokens_without_newlines


def _generate_tokens_without_newlines(readline):
    for tok in _tokenize.generate_tokens(readline):
        if tok[0] in (_tokenize.NEWLINE, _tokenize.NL):
            continue
        yield tok


def _load_tempita():
    d = os.path.dirname(Cython.Tempita.__file__)
    pkg = types.ModuleType("oracle_tempita")
    pkg.__path__ = [d]
    sys.modules["oracle_tempita"] = pkg
    mods = {}
    for name in ("_looper", "_tempita"):
        spec = importlib.util.spec_from_file_location(
            "oracle_tempita." + name, os.path.join(d, name + ".py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules["oracle_tempita." + name] = mod
        spec.loader.exec_module(mod)
        mods[name] = mod
    mods["_tempita"].tokenize = _TokenizeWithoutNewlines()
    return mods["_tempita"]


def _list_zip(*args):
    return list(zip(*args))


def main(src, dst, **params):
    tempita = _load_tempita()
    with open(src) as f:
        text = f.read()
    # The templates were written for Python 2, where zip() returns a list
    # that can be iterated more than once (src/butterfly.c.in:31-36 iterates
    # nvecs_instances once per scatter group).
    out = tempita.sub(text, zip=_list_zip, **params)
    with open(dst, "w") as f:
        f.write("/* generated from %s by oracle/expand_tempita.py */\n" % src)
        f.write(out)


if __name__ == "__main__":
    # template parameters as name=python-literal pairs (the instantiation
    # arguments of wavemoth/cuda/legendre_transform.py:23-33 for the GPU kernel)
    import ast
    params = dict((k, ast.literal_eval(v)) for k, v in (a.split("=", 1) for a in sys.argv[3:]))
    main(sys.argv[1], sys.argv[2], **params)
