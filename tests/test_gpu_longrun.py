"""Long-run statistics against the oracle: the flow is chaotic, so step-wise
fields drift apart at the rounding level and grow, but time averages must
agree.  The bar is the one stated for full runs: time-averaged velocity and
per-turbine thrust / power within 1e-3 relative.  Run here on the 40x20x20
two-turbine log-law case for 1000 steps, averaging over steps 101-1000, in
the fast (default) mode (measured over 300 steps: 1e-9 relative)."""
import numpy as np
import pytest

from conftest import package
import oracle as O
from test_gpu_parity import rel

pytestmark = pytest.mark.gpu

STEPS, AVG_FROM = 1000, 101
BAR = 1e-3


def test_time_averages_over_300_steps(make_case):
    pkg = package()
    spec, mesh, d, U0, prof = make_case("tiny-loglaw", steps=STEPS,
                                        tavg_start_time=AVG_FROM * 1e-3)
    s = pkg.Solver(d)
    o = O.CRestatement(d)
    for x in (s, o):
        x.set_inflow_profile(prof)
        x.set_state(U0)
    sums = {"gpu": None, "oracle": None}
    n_avg = 0
    for step in range(STEPS + 1):
        s.step(1)
        o.step(1)
        if step >= AVG_FROM:
            # power = torque |Omega| with a fixed rotor speed: torque stands for it
            th, tq, _ = s.turbines()
            tqo, tho = o.turbines()
            a = np.concatenate([th, tq])
            b = np.concatenate([tho, tqo])
            sums["gpu"] = a if sums["gpu"] is None else sums["gpu"] + a
            sums["oracle"] = b if sums["oracle"] is None else sums["oracle"] + b
            n_avg += 1
    mean_g, mean_o = sums["gpu"] / n_avg, sums["oracle"] / n_avg
    err = np.abs(mean_g - mean_o) / np.abs(mean_o)
    print("time-averaged thrust, torque (GPU / oracle):", mean_g, mean_o, "rel", err)
    assert np.all(err <= BAR), err
    r = rel(s.field("Utavg"), o.field("Utavg"))
    print("time-averaged velocity rel L2", r)
    assert r <= BAR
