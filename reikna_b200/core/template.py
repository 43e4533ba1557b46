"""A small renderer for the template syntax reikna's transformation snippets use.

reikna writes transformation and kernel code as Mako templates
(reikna/core/transformation_modules.py, examples/demo_fftshift_transformation.py:42-67).
Mako itself is not a dependency here; this module renders the subset those snippets
use, with the same meaning:

* ``${expression}``: the value of a Python expression, as text;
* ``<% statements %>``: Python statements (names they bind stay visible below);
* control lines ``% for ...:`` / ``% endfor``, ``% if ...:`` / ``% elif ...:`` /
  ``% else:`` / ``% endif``, ``% while ...:`` / ``% endwhile`` (leading whitespace
  allowed; ``%%`` at a line start is a literal ``%``);
* ``## comment`` lines are dropped, and a backslash right before a newline joins the
  two lines.

The template compiles to Python source once (cached by text) and renders against a
namespace of keyword arguments.
"""

from __future__ import annotations

import functools
import textwrap


class TemplateError(ValueError):
    pass


def _find_close(text: str, pos: int) -> int:
    """Index of the ``}`` closing the ``${`` whose body starts at ``pos`` (nested
    braces and string literals respected)."""
    depth, i, quote = 1, pos, None
    while i < len(text):
        c = text[i]
        if quote:
            if c == "\\":
                i += 2
                continue
            if text.startswith(quote, i):
                i += len(quote)
                quote = None
                continue
        elif c in "'\"":
            quote = text[i : i + 3] if text[i : i + 3] in ("'''", '"""') else c
            i += len(quote)
            continue
        elif c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                return i
        i += 1
    raise TemplateError("unterminated ${...} expression")


def _tokens(text: str):
    i, n = 0, len(text)
    buf = []

    def flush():
        if buf:
            yield ("text", "".join(buf))
            buf.clear()

    while i < n:
        line_start = i == 0 or text[i - 1] == "\n"
        if line_start:
            j = i
            while j < n and text[j] in " \t":
                j += 1
            if text.startswith("##", j):
                e = text.find("\n", j)
                i = n if e < 0 else e + 1
                continue
            if j < n and text[j] == "%" and not text.startswith("%%", j) and not text.startswith("%>", j):
                yield from flush()
                e = text.find("\n", j)
                line = text[j + 1 : (n if e < 0 else e)]
                yield ("control", line.strip())
                i = n if e < 0 else e + 1
                continue
            if text.startswith("%%", j):
                buf.append(text[i:j] + "%")
                i = j + 2
                continue
        if text.startswith("<%", i) and not text.startswith("<%def", i) and not text.startswith("<%include", i):
            yield from flush()
            start = i + 3 if text.startswith("<%!", i) else i + 2
            e = text.find("%>", start)
            if e < 0:
                raise TemplateError("unterminated <% ... %> block")
            yield ("code", text[start:e])
            i = e + 2
            continue
        if text.startswith("${", i):
            yield from flush()
            e = _find_close(text, i + 2)
            yield ("expr", text[i + 2 : e].strip())
            i = e + 1
            continue
        if text.startswith("\\\n", i):
            i += 2
            continue
        buf.append(text[i])
        i += 1
    yield from flush()


@functools.lru_cache(maxsize=256)
def _compile(text: str):
    lines = []
    indent = 0

    def emit(s: str):
        lines.append("    " * indent + s)

    for kind, val in _tokens(text):
        if kind == "text":
            emit(f"__out.append({val!r})")
        elif kind == "expr":
            emit(f"__out.append(str({val}))")
        elif kind == "code":
            body = textwrap.dedent(val.strip("\n"))
            for ln in body.splitlines():
                if ln.strip():
                    emit(ln)
        else:
            word = val.split(None, 1)[0].rstrip(":") if val else ""
            if word.startswith("end"):
                indent -= 1
                if indent < 0:
                    raise TemplateError(f"unbalanced '% {val}'")
                continue
            if word in ("elif", "else", "except", "finally"):
                indent -= 1
                emit(val if val.endswith(":") else val + ":")
                indent += 1
                continue
            emit(val if val.endswith(":") else val + ":")
            indent += 1
    if indent != 0:
        raise TemplateError("a control block is not closed")
    src = "\n".join(lines) if lines else "pass"
    try:
        return compile(src, "<template>", "exec")
    except SyntaxError as e:
        raise TemplateError(f"template code does not compile: {e}\n{src}") from e


def render(text: str, **namespace) -> str:
    """Render ``text`` with the names in ``namespace``."""
    code = _compile(text)
    ns = dict(namespace)
    out = []
    ns["__out"] = out
    exec(code, ns)  # noqa: S102 - templates are the caller's own code, as with Mako
    return "".join(out)
