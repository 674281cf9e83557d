"""Case generator: mesh rules, PRNG, JSON contract (CPU only)."""
import json
import math

import numpy as np

from conftest import casegen
import oracle as O


def test_splitmix64_known_answers():
    cg = casegen()
    # published first outputs of splitmix64 seeded with 0
    got = [int(v) for v in cg.splitmix64(0, 3)]
    assert got == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_gaussian_is_deterministic_and_standard():
    cg = casegen()
    a, b = cg.gaussian(3, 200001), cg.gaussian(3, 200001)
    np.testing.assert_array_equal(a, b)
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1) < 0.01
    assert not np.array_equal(cg.gaussian(0, 10), cg.gaussian(1, 10))


def test_stretched_mesh_rules():
    cg = casegen()
    m = cg.make_mesh(32, 16, 64)
    gc = m.gc
    dz = np.diff(0.5 * (m.z[gc:-gc][1:] + m.z[gc:-gc][:-1]))
    nodes, beta = cg.tanh_wall_nodes(64, 5.0)
    d = np.diff(nodes)
    assert np.max(d[1:] / d[:-1]) <= 1.05 + 1e-9
    assert d[0] < d[-1]                       # clustered toward z = 0
    assert nodes[0] == 0.0 and nodes[-1] == 5.0
    # guide cells follow x[i] = 3x[i+1] - 3x[i+2] + x[i+3] (script/convertmesh.py:22-32)
    for c in (m.x, m.y, m.z):
        assert math.isclose(c[1], 3 * c[2] - 3 * c[3] + c[4], rel_tol=0, abs_tol=1e-12)
        assert math.isclose(c[-2], 3 * c[-3] - 3 * c[-4] + c[-5], rel_tol=0, abs_tol=1e-12)
    assert len(dz) > 0


def test_case_files_follow_reference_contract(tmp_path):
    cg = casegen()
    spec = cg.config("c4", n=(32, 16, 16))
    cg.write_case(spec, str(tmp_path))
    s = json.load(open(tmp_path / "setup.json"))
    assert s["eq"]["method"] == "BiCG" and s["eq"]["preconditioner"]["method"] == "Jacobi"
    yaws = [t["angle"][2] for t in s["windturbine array"]]
    assert yaws[0] == {"amp": 0, "T": 1, "phase": 0, "offset": 0} and yaws[1] == 10.0
    wt = json.load(open(tmp_path / "windturbine.json"))
    assert wt["blade"]["attack angle"][0] == -180.0 and len(wt["blade"]["attack angle"]) == 721
    c = O.Case(str(tmp_path))
    assert c.max_step == spec.steps
    assert [t["type"] for t in c.turbines] == ["yaw", "yaw", "yaw"]
    assert math.isclose(c.turbines[1]["formula"][3], math.radians(10.0))


def test_polar_and_profile():
    cg = casegen()
    atk, cd, cl = cg.polar_tables()
    i0 = int(np.argmin(np.abs(atk)))
    assert cl[i0] == 0.0 and math.isclose(cd[i0], 0.01)
    assert math.isclose(cl.max(), 2 * math.pi * math.radians(15.0))
    spec = cg.config("c4", n=(16, 8, 8))
    mesh = cg.make_mesh(*spec.n)
    prof = cg.inflow_profile(spec, mesh)
    k = mesh.gc + 3
    assert math.isclose(prof[4, k, 0], (0.05 / 0.41) * math.log(mesh.z[k] / 1e-3))
    U = cg.initial_velocity(spec, mesh)
    assert np.all(U[0] == prof[None, :, :, :][0])    # guide cells untouched by the noise


def test_command_line_time_step(tmp_path):
    """`python -m 3dalm_b200.casegen <config> <dir> --dt` sets the case's
    time step (the benchmark's 5e-4 on the 512x256x128 configuration) and
    runtime.time = steps * dt."""
    cg = casegen()
    d = str(tmp_path / "case")
    cg.main(["tiny-loglaw", d, "--dt", "5e-4", "--steps", "3", "--no-state"])
    setup = json.load(open(f"{d}/setup.json"))
    text = json.dumps(setup)
    assert '"dt": 0.0005' in text
    assert math.isclose(setup["runtime"]["time"], 3 * 5e-4)
