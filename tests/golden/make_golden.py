"""Generate tests/golden/reference_tiny.npz from the REFERENCE solver itself.

The reference (ki2098/3dalm) ships no golden vectors, so these fixtures are
outputs of its own FP64 code, compiled from its sources by oracle/Makefile
into oracle/_ref/libref3dalm.so, on small synthetic cases written by
3dalm_b200/casegen.py.  They let the CPU tests pin the C restatement
(oracle/dalm_oracle.c) when the reference sources are not available.

Run from the repository root (needs the reference sources for `make ref`):
    python tests/golden/make_golden.py
"""
import importlib
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

cg = importlib.import_module("3dalm_b200.casegen")

# (case name, turbine overrides (yaw, pitch, omega) or None, steps)
CASES = [
    ("tiny-sor", None, 5),
    ("tiny-bicg", None, 5),
    ("tiny-sorpc", None, 5),
    ("tiny-turbine", None, 5),
    ("tiny-loglaw", None, 5),
    ("tiny-turbine", ([7.5], [2.0], [10.0]), 5),
]
FIELDS = ("U", "JU", "p", "nut", "div", "f", "b")
SAMPLE_STRIDE = 97


def checksums(a: np.ndarray) -> np.ndarray:
    """sum, sum of squares and a sin-weighted sum of the flattened array."""
    v = a.reshape(-1)
    w = np.sin(np.arange(v.size, dtype=np.float64) * 0.7071)
    return np.array([v.sum(), (v * v).sum(), (v * w).sum()])


def case_key(name, params):
    return name + ("-params" if params else "")


def run_case(name, params, steps, tmp):
    spec = cg.config(name)
    d = os.path.join(tmp, case_key(name, params))
    mesh = cg.write_case(spec, d)
    U0 = cg.initial_velocity(spec, mesh)
    prof = cg.inflow_profile(spec, mesh)
    ref = O.Reference(d)
    if prof is not None:
        ref.set_inflow_profile(prof)
    if params:
        ref.set_turbine_params(*params)
    ref.set_state(U0)
    rec = {}
    stats, turb = [], []
    for _ in range(steps):
        ref.step(1)
        s = ref.stats()
        stats.append([s["step"], s["it"], s["err"], s["avg_div"], s["max_cfl"]])
        tq, th = ref.turbines()
        turb.append(np.concatenate([tq, th]) if tq.size else np.zeros(0))
    key = case_key(name, params)
    rec[key + "/stats"] = np.array(stats, dtype=np.float64)
    rec[key + "/turbines"] = np.array(turb, dtype=np.float64)
    for f in FIELDS:
        a = ref.field(f)
        rec[key + "/" + f + "/checksums"] = checksums(a)
        rec[key + "/" + f + "/sample"] = a.reshape(-1)[::SAMPLE_STRIDE].copy()
    if ref.turbine_count():
        r, dr, ch, tw, cd, cl, atk = ref.point_tables()
        rec[key + "/point_tables"] = np.concatenate([r, dr, ch, tw, cd.reshape(-1)[::7],
                                                     cl.reshape(-1)[::7]])
    ref.close()
    return rec


def main():
    O.build(ref=True)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, params, steps in CASES:
            out.update(run_case(name, params, steps, tmp))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_tiny.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
