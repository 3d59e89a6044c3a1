"""Reader for the reference's `.sim` block scripts.

Same syntax and accessors as SCRIPT_READER / SCRIPT_BLOCK
(SCRIPT_READER.h:161-173, SCRIPT_READER.cpp): named blocks in braces,
`key = value` assignments with numbers, booleans, quoted strings and
parenthesised 2/3/4-vectors, `//` and `/* */` comments.  Every getter takes a
default that is returned when the key is absent, as the reference's do.
Numbers follow the reference's syntax (no exponent); a value that does not
parse is rejected instead of being silently truncated.
"""
import re

_TOKEN = re.compile(r'\s*(?:(//[^\n]*|/\*.*?\*/)|("[^"]*")|(\([^)]*\))|([{}=])|([^\s{}=()"]+))', re.S)


class ScriptError(ValueError):
    pass


class SCRIPT_BLOCK:
    def __init__(self, name="", values=None, blocks=None):
        self.name = name
        self.values = values or {}
        self.blocks = blocks or []

    # accessors mirroring SCRIPT_BLOCK::Get* -------------------------------
    def FindBlock(self, name):
        for b in self.blocks:
            if b.name == name:
                return b
        return SCRIPT_BLOCK(name)

    def FindBlocks(self, name):
        return [b for b in self.blocks if b.name == name]

    def _raw(self, key):
        return self.values.get(key)

    def GetFloat(self, key, default=0.0):
        v = self._raw(key)
        if v is None:
            return float(default)
        return _number(v, key)

    def GetInteger(self, key, default=0):
        v = self._raw(key)
        if v is None:
            return int(default)
        return int(_number(v, key))

    def GetBoolean(self, key, default=False):
        v = self._raw(key)
        if v is None:
            return bool(default)
        if v not in ("true", "false"):
            raise ScriptError(f"{key}: expected true/false, got {v!r}")
        return v == "true"

    def GetString(self, key, default=""):
        v = self._raw(key)
        if v is None:
            return default
        return v[1:-1] if v.startswith('"') else v

    def GetVector3(self, key, default=(0.0, 0.0, 0.0)):
        v = self._raw(key)
        if v is None:
            return tuple(float(a) for a in default)
        parts = [p.strip() for p in v.strip("()").split(",")]
        if len(parts) != 3:
            raise ScriptError(f"{key}: expected a 3-vector, got {v!r}")
        return tuple(_number(p, key) for p in parts)

    def GetVector3Int(self, key, default=(0, 0, 0)):
        return tuple(int(a) for a in self.GetVector3(key, default))


_LINE_COMMENT = object()
_NUM = re.compile(r"^-*\d*\.*\d+$")


def _number(text, key):
    t = text.strip()
    if not _NUM.match(t):
        raise ScriptError(f"{key}: {text!r} is not a number in the script syntax (digits, one '.', no exponent)")
    neg = t.count("-") % 2 == 1
    return -float(t.lstrip("-")) if neg else float(t.lstrip("-"))


def _skip_block(tokens, pos):
    depth = 0
    while pos < len(tokens):
        if tokens[pos] == "{":
            depth += 1
        elif tokens[pos] == "}":
            depth -= 1
            if depth == 0:
                return pos + 1
        pos += 1
    raise ScriptError("commented-out block is not closed")


def _parse(tokens, pos, name):
    block = SCRIPT_BLOCK(name)
    while pos < len(tokens):
        tok = tokens[pos]
        if tok is _LINE_COMMENT:
            # "// NAME {" comments out the whole block (SCRIPT_READER.cpp:301-330)
            pos += 1
            if pos < len(tokens) and tokens[pos] == "{":
                pos = _skip_block(tokens, pos)
            continue
        if tok == "}":
            return block, pos + 1
        if pos + 1 < len(tokens) and tokens[pos + 1] == "{":
            child, pos = _parse(tokens, pos + 2, tok)
            block.blocks.append(child)
            continue
        if pos + 2 < len(tokens) and tokens[pos + 1] == "=":
            block.values[tok] = tokens[pos + 2]
            pos += 3
            continue
        raise ScriptError(f"unexpected token {tok!r} in block {name!r}")
    if name:
        raise ScriptError(f"block {name!r} is not closed")
    return block, pos


class SCRIPT_READER:
    """Parses a .sim file (or text) into a root SCRIPT_BLOCK."""

    def __init__(self, path=None, text=None):
        if text is None:
            with open(path) as f:
                text = f.read()
        tokens = []
        for m in _TOKEN.finditer(text):
            if m.group(1):
                if m.group(1).startswith("//"):
                    tokens.append(_LINE_COMMENT)
                continue
            tok = m.group(2) or m.group(3) or m.group(4) or m.group(5)
            if tok:
                tokens.append(tok)
        self.root, _ = _parse(tokens, 0, "")

    def FindBlock(self, name):
        return self.root.FindBlock(name)
