"""Writes tests/golden/oracle_states.npz: states of the FP64 oracle
(oracle/shyref.cpp, the CPU restatement of the reference's step) after a
fixed number of steps of two seeded cases, as fixtures the parity tests
compare against without running the oracle:

* the 2D tidal channel (one layer, M2 0.5 m, dt 60 s), 60 steps;
* the small 3D basin of the parity tests (about 1500 nodes, 12 z-layers,
  wind, M2, T/S with baroclinic pressure, dt 120 s), 20 steps.

Values are stored in FP32 (what the GPU state holds), which keeps the file
small; the oracle's own regression check compares at FP32 resolution.

    python tests/golden/make_golden.py

The reference itself is Fortran and no Fortran compiler exists here, so
these are the oracle's outputs; tests/test_oracle_golden.py checks that
the oracle still reproduces them."""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT / "shyfemcm-ismar_b200"), str(ROOT / "oracle")]

# (name, constructor in shygpu.cases, its arguments, steps, fields kept)
CASES = [
    ("channel", "channel_case", {}, 60, ("znv", "utlnv", "vtlnv")),
    ("basin3d_small", "basin3d_case", {"nkn_target": 1500, "nlv": 12}, 20,
     ("znv", "utlnv", "vtlnv", "tempv", "saltv", "wlnv", "hdknv")),
]
OUT = HERE / "oracle_states.npz"


def make_case(ctor, args):
    from shygpu import cases
    return getattr(cases, ctor)(**args)


def oracle_states():
    import shyref
    out = {}
    for name, ctor, args, steps, fields in CASES:
        o = shyref.OracleModel(make_case(ctor, args))
        o.run(steps)
        st = o.state()
        for f in fields:
            out[f"{name}/{f}"] = np.asarray(st[f], np.float32)
    return out


def main():
    arrays = oracle_states()
    meta = json.dumps([{"name": n, "ctor": c, "args": a, "steps": s, "fields": list(f)} for n, c, a, s, f in CASES])
    np.savez_compressed(OUT, meta=np.array(meta), **arrays)
    print(OUT, sum(v.nbytes for v in arrays.values()), "bytes of state")


if __name__ == "__main__":
    main()
