"""The GPU ground-state producer (bdg_ground_state: split-step imaginary time,
then bordered Newton steps) against the oracle's (oracle.itp_ground_state +
oracle.newton_polish), through the committed fixtures tests/golden/gs16.npz,
c1_32.npz and c2_64.npz that the oracle produced.  Both stop the imaginary
time at the same rule (|d mu| < 1e-12 per step, dt = 1e-3) and polish to the
exact discrete stationary state, so the polished states must agree to the
rounding of the Newton solves."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_fixtures as FX  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["gs16", "c1_32", "c2_64"])
def test_gpu_ground_state_matches_oracle_fixture(bdg, name):
    from bdg_lobpcg_b200 import problems

    f = FX.load(name)
    cfg = dict(N=[int(v) for v in f["N"]], L=[float(v) for v in f["L"]],
               omegas=tuple(float(v) for v in f["omegas"]), g=float(f["g"]), gdd=float(f["gdd"]),
               rc=float(f["rc"]))
    psi, mu, steps, stationarity, _ = problems.ground_state(bdg, cfg)
    ref = f["psi"]
    assert stationarity < 1e-12, stationarity
    assert abs(mu - float(f["mu"])) <= 1e-11 * abs(float(f["mu"])), (mu, float(f["mu"]))
    # the imaginary-time phase stops by the same rule (a step or two apart by rounding)
    assert abs(steps - int(f["steps"])) <= 5, (steps, int(f["steps"]))
    err = float(np.max(np.abs(psi - ref)) / np.max(np.abs(ref)))
    assert err < 1e-9, err
