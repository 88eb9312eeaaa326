"""Regenerate ``reference_vectors.json`` from the reference's own test vectors.

Usage: ``python make_golden.py REFERENCE_ROOT`` (or set ``YM_REFERENCE_ROOT``),
where REFERENCE_ROOT is a read-only checkout of the reference repository.
Machines without that checkout run the tests from the JSON this script
writes.  It copies, unchanged,
the reference's ``test-vectors/*.json`` files that pin the hot path, plus the
literal golden values the reference's Rust tests assert
(``tests/su3_ensemble.rs``, ``tests/su2_ensemble.rs``,
``reference/rust/src/glueball_*.rs``), which the JSON vectors duplicate.
"""
import json
import os
import sys

FILES = [
    "su2-ensemble-v1.json",
    "su2-observables-v1.json",
    "su2-wilson-v1.json",
    "su3-algebra-v1.json",
    "su3-lattice-v1.json",
    "su3-ensemble-v1.json",
    "path-holonomy-v1.json",
    "glueball-operators-phase3a-v1.json",
    "glueball-spatial-stout-phase3b1-v1.json",
    "glueball-spatial-block-phase3b2-v1.json",
    "glueball-connected-correlator-phase3c-v1.json",
    "glueball-effective-mass-phase3d-v1.json",
    "glueball-scalar-fit-phase3e-v1.json",
    "glueball-scalar-variational-phase3j-v1.json",
    "glueball-scalar-production-phase3f-v1.json",
    "sampling-efficiency-v1.json",
    "su3-plaquette-baseline-v1.json",
    "su3-plaquette-baseline-v2.json",
    "su2-plaquette-baseline-v1.json",
]


def main() -> int:
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("YM_REFERENCE_ROOT")
    if not root:
        print("usage: make_golden.py REFERENCE_ROOT (or set YM_REFERENCE_ROOT)", file=sys.stderr)
        return 2
    out = {"source": "QSOLKCB/YANG-MILLS test-vectors", "vectors": {}}
    for name in FILES:
        with open(os.path.join(root, "test-vectors", name)) as fh:
            out["vectors"][name] = json.load(fh)
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "reference_vectors.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
        fh.write("\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
