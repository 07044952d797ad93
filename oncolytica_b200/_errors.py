"""CompilationError (reference framework/src/oncolytica/core/utils/_errors.py:9-19)."""
from __future__ import annotations

import ast


class CompilationError(Exception):
    """A rule cannot be compiled to CUDA; carries the offending AST node."""

    def __init__(self, message: str, node: ast.AST | None = None, source: str | None = None,
                 filename: str | None = None, line_offset: int = 0) -> None:
        self.node = node
        self.raw_message = message
        loc = ""
        if node is not None and getattr(node, "lineno", None) is not None:
            line = node.lineno + line_offset
            loc = f" (line {line}" + (f" of {filename}" if filename else "") + ")"
            if source:
                lines = source.splitlines()
                if 0 < node.lineno <= len(lines):
                    loc += "\n    " + lines[node.lineno - 1].strip()
        super().__init__(message + loc)
