"""ym_status codes as Python exceptions.

The reference reports failures through fail-closed Rust enums
(``ReferenceError`` lib.rs:52-73, ``Su3EnsembleError`` su3_ensemble.rs:123-137,
...).  The C ABI flattens them to the int32 codes of ``include/ym_status.h``;
here each code becomes a ``YmError`` whose ``variant`` is the reference
variant name in CamelCase (``YM_ERR_BETA_OUTSIDE_REFERENCE_RANGE`` ->
``BetaOutsideReferenceRange``), so callers can match on the same names the
reference's tests use.
"""
from __future__ import annotations

import os
import re

_HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))),
                    "include", "ym_status.h")


def _load_codes() -> dict:
    codes = {}
    with open(_HDR) as fh:
        for m in re.finditer(r"YM_ERR_([A-Z0-9_]+)\s*=\s*(\d+)", fh.read()):
            name = "".join(part.capitalize() for part in m.group(1).split("_"))
            codes[int(m.group(2))] = name
    return codes


CODES = _load_codes()
VARIANTS = {v: k for k, v in CODES.items()}


class YmError(RuntimeError):
    """A nonzero ym_status from libymgpu."""

    def __init__(self, code: int, where: str, cuda_error: int = 0):
        self.code = code
        self.variant = CODES.get(code, f"Unknown{code}")
        self.cuda_error = cuda_error
        extra = f" (cudaError {cuda_error})" if code == VARIANTS.get("Cuda") else ""
        super().__init__(f"{where}: {self.variant}{extra}")


def check(code: int, where: str) -> None:
    if code != 0:
        cuda = 0
        if code == VARIANTS.get("Cuda"):
            from ._lib import lib
            cuda = lib().ym_last_cuda_error()
        raise YmError(code, where, cuda)
