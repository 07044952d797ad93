"""Rule translator: Python rule DSL -> CUDA C compiled by NVRTC for sm_100a.

Replaces the reference's WGSL translator
(framework/src/oncolytica/gpu/compiler/_compiler.py, _shader_builder.py,
translator/_stmt_translator.py, translator/_expr_translator.py).
"""
from oncolytica_b200.compiler.emit_cuda import ModelLayout, Program, translate_model

__all__ = ["ModelLayout", "Program", "translate_model"]
