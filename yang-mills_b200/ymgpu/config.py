"""Canonical text configurations and ensemble checkpoints.

``su2_to_canonical_config`` / ``su2_from_canonical_config`` are the
reference's ``Lattice4::to_canonical_config`` / ``from_canonical_config``
(lib.rs:587-694, format YM-SU2-CONFIG-V1) byte for byte; the ``su3_`` pair
is the same format for SU(3) links (YM-SU3-CONFIG-V1, include/ym_config.h).
Both run in libymgpu's host code.

A checkpoint is every chain of an ``Ensemble`` in that text plus what the
counter-based streams need to continue: each chain's beta and seed and the
ensemble's sweep index.  Because every link update draws its random words
from (seed, sweep index, site, direction) alone, a chain restored from a
checkpoint continues bit for bit as if it had never stopped.
"""
from __future__ import annotations

import ctypes as C
import struct
from typing import Tuple

import numpy as np

from . import _lib as L
from ._lib import lib
from .errors import VARIANTS, YmError, check

SU2_CONFIG_FORMAT_ID = "YM-SU2-CONFIG-V1"
SU3_CONFIG_FORMAT_ID = "YM-SU3-CONFIG-V1"
CHECKPOINT_FORMAT_ID = "YM-B200-CHECKPOINT-V1"

_WORDS = {"su2": 4, "su3": 18}


def _encode(group: str, extents, links, lift: bool) -> str:
    ext = (C.c_int64 * 4)(*[int(e) for e in extents])
    arr = np.ascontiguousarray(np.asarray(links, dtype=np.complex128 if group == "su3" else np.float64))
    flat = arr.view(np.float64).reshape(-1)
    # the library reads words x links values once the extents pass its checks
    if all(int(e) >= 2 for e in extents) and flat.size != _WORDS[group] * _link_count(extents):
        raise YmError(VARIANTS["InvalidArgument"], f"{group}_to_canonical_config")
    fn = getattr(lib(), f"ym_{group}_to_canonical_config")
    n = C.c_int64()
    check(fn(ext, flat.ctypes.data_as(L.P(L.f64)), int(lift), None, 0, C.byref(n)),
          f"{group}_to_canonical_config")
    buf = C.create_string_buffer(n.value)
    check(fn(ext, flat.ctypes.data_as(L.P(L.f64)), int(lift), buf, n.value, C.byref(n)),
          f"{group}_to_canonical_config")
    return buf.raw[:n.value].decode("ascii")


def _link_count(extents) -> int:
    return int(np.prod([int(e) for e in extents])) * 4


def _decode(group: str, text, lift: bool):
    raw = text.encode("utf-8") if isinstance(text, str) else bytes(text)
    fn = getattr(lib(), f"ym_{group}_from_canonical_config")
    ext = (C.c_int64 * 4)()
    check(fn(raw, len(raw), int(lift), ext, None, 0), f"{group}_from_canonical_config")
    n = _link_count(ext)
    flat = np.zeros(n * _WORDS[group])
    check(fn(raw, len(raw), int(lift), ext, flat.ctypes.data_as(L.P(L.f64)), n),
          f"{group}_from_canonical_config")
    links = flat.reshape(n, 4) if group == "su2" else flat.view(np.complex128).reshape(n, 3, 3)
    return tuple(int(e) for e in ext), links


def su2_to_canonical_config(extents, links, lift_reference_caps: bool = False) -> str:
    """Lattice4::to_canonical_config (lib.rs:587-616); links [L][4]."""
    return _encode("su2", extents, links, lift_reference_caps)


def su2_from_canonical_config(text, lift_reference_caps: bool = False) -> Tuple[tuple, np.ndarray]:
    """Lattice4::from_canonical_config (lib.rs:618-694) -> (extents, links [L][4])."""
    return _decode("su2", text, lift_reference_caps)


def su3_to_canonical_config(extents, links, lift_reference_caps: bool = False) -> str:
    """YM-SU3-CONFIG-V1 of an SU(3) lattice; links [L][3][3] complex."""
    return _encode("su3", extents, links, lift_reference_caps)


def su3_from_canonical_config(text, lift_reference_caps: bool = False) -> Tuple[tuple, np.ndarray]:
    """-> (extents, links [L][3][3] complex128)."""
    return _decode("su3", text, lift_reference_caps)


def _bits(x: float) -> str:
    return "%016x" % struct.unpack("<Q", struct.pack("<d", float(x)))[0]


def _unbits(s: str) -> float:
    return struct.unpack("<d", struct.pack("<Q", int(s, 16)))[0]


def save_checkpoint(ens, path: str) -> None:
    """Every chain of an FP64 ``Ensemble`` (SU(2) or SU(3)) with its beta,
    seed and the sweep index, so ``load_checkpoint`` resumes the streams.
    Two-row FP32 storage is refused (its links are not SU(3) to 5e-12)."""
    from .ensemble import F64, SU2
    if ens.precision != F64:
        raise YmError(VARIANTS["UnsupportedPrecision"], "save_checkpoint")
    group = "su2" if ens.group == SU2 else "su3"
    parts = [f"{CHECKPOINT_FORMAT_ID}\ngroup={group}\nchains={ens.n_chains}\n"
             f"sweep_index={ens.sweep_index}\n"]
    for k in range(ens.n_chains):
        text = _encode(group, ens.extents[k], ens.download(k), True)
        parts.append(f"chain={k} beta={_bits(ens.beta[k])} seed={int(ens.seeds[k]):016x} "
                     f"bytes={len(text)}\n")
        parts.append(text)
    with open(path, "w", newline="\n") as fh:
        fh.write("".join(parts))


def load_checkpoint(path: str, device: int = 0):
    """The ``Ensemble`` a checkpoint holds, positioned at its sweep index."""
    from .ensemble import SU2, SU3, Ensemble
    with open(path, "r", newline="\n") as fh:
        data = fh.read()
    bad = YmError(VARIANTS["InvalidConfigurationEncoding"], "load_checkpoint")
    head = data.split("\n", 4)
    if len(head) < 5 or head[0] != CHECKPOINT_FORMAT_ID:
        raise bad
    try:
        group = head[1].removeprefix("group=")
        n = int(head[2].removeprefix("chains="))
        sweep = int(head[3].removeprefix("sweep_index="))
    except ValueError:
        raise bad from None
    if group not in _WORDS or n <= 0 or not head[1].startswith("group=") or sweep < 0:
        raise bad
    rest = head[4]
    extents, betas, seeds, lattices = [], [], [], []
    for k in range(n):
        line, _, rest = rest.partition("\n")
        fields = dict(f.split("=", 1) for f in line.split(" ") if "=" in f)
        if fields.get("chain") != str(k) or not {"beta", "seed", "bytes"} <= set(fields):
            raise bad
        size = int(fields["bytes"])
        text, rest = rest[:size], rest[size:]
        ext, links = _decode(group, text, True)
        extents.append(ext)
        betas.append(_unbits(fields["beta"]))
        seeds.append(int(fields["seed"], 16))
        lattices.append(links)
    if rest:
        raise bad
    ens = Ensemble(extents, betas, seeds, group=SU2 if group == "su2" else SU3,
                   lift_reference_caps=True, device=device)
    for k, links in enumerate(lattices):
        ens.upload(k, links)
    ens.sweep_index = sweep
    return ens
