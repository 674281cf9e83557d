"""The multi-rank CPU baseline (oracle/_ref/ref_mpirun): the reference's own
time step as N MPI ranks over the shared-memory MPI subset
(oracle/ref_shim/shm/mpi.h).  Split into x-slabs, every rank exchanges halos
and reduces its dots through the MPI calls, so a broken exchange shows up as
a wrong iteration count or residual.  Checked against the single-rank oracle
(the C restatement) on the same case: the Poisson iteration counts agree
within the summation-order envelope (the ranks sum their slabs separately,
as the reference does under MPI) and every solve meets the tolerance."""
import json
import os
import subprocess

import pytest

from conftest import ROOT, casegen
import oracle as O

BIN = os.path.join(ROOT, "oracle", "_ref", "ref_mpirun")

pytestmark = pytest.mark.skipif(not os.path.exists(BIN), reason="ref_mpirun not built")


def run_ranks(d, spec, ranks, warmup, steps):
    cg = casegen()
    out = os.path.join(d, f"r{ranks}.json")
    cmd = [BIN, d, "--ranks", str(ranks), "--warmup", str(warmup), "--steps", str(steps),
           "--out", out, "--state", os.path.join(d, cg.STATE_FILE)]
    if os.path.exists(os.path.join(d, cg.PROFILE_FILE)):
        cmd += ["--profile", os.path.join(d, cg.PROFILE_FILE)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    with open(out) as f:
        return json.load(f)


@pytest.mark.parametrize("name", ["tiny-bicg", "tiny-loglaw", "tiny-sor"])
def test_ranks_match_single_rank_oracle(tmp_path, name):
    cg = casegen()
    spec = cg.config(name)
    d = str(tmp_path / name)
    mesh = cg.write_case(spec, d)
    cg.write_state_files(spec, mesh, d)
    o = O.CRestatement(d)
    prof = cg.inflow_profile(spec, mesh)
    if prof is not None:
        o.set_inflow_profile(prof)
    o.set_state(cg.initial_velocity(spec, mesh))
    o.step(1)
    ref_its = []
    for _ in range(4):
        o.step(1)
        ref_its.append(o.stats()["it"])
    o.close()
    for ranks in (1, 2, 3):
        res = run_ranks(d, spec, ranks, 1, 4)
        assert res["ranks"] == ranks and res["steps"] == 4
        assert res["cells"] == spec.n[0] * spec.n[1] * spec.n[2]
        for a, b in zip(res["iterations"], ref_its):
            assert abs(a - b) <= max(3, 0.25 * b), (ranks, res["iterations"], ref_its)
        if spec.solver == "BiCG":
            assert max(res["residuals"]) <= spec.tol, (ranks, res["residuals"])
        assert all(t > 0 for t in res["step_seconds"])


def test_rank_failure_is_reported(tmp_path):
    """A rank that cannot read its input exits non-zero; the launcher stops
    the other ranks and reports failure instead of waiting for them."""
    cg = casegen()
    spec = cg.config("tiny-bicg")
    d = str(tmp_path / "bad")
    cg.write_case(spec, d)
    cmd = [BIN, d, "--ranks", "2", "--warmup", "0", "--steps", "1", "--out",
           os.path.join(d, "r.json"), "--state", os.path.join(d, "missing.f64")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert not os.path.exists(os.path.join(d, "r.json"))
