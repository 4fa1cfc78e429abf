"""The velocity step on a real flow state written by the reference solver
(tests/golden/particle_state_00500_sub8.csv), through the reference-shaped
caller: state file -> Particle -> VelocityCalc.get_velocity, against the
oracle (plain form) and the FP64 direct sum (mixed form)."""
import os

import numpy as np
import pytest

from lsmps_vpm_v2_b200 import PREC_MIXED, Particle, VelocityCalc, default_params, read_particle_state
from lsmps_vpm_v2_b200.workloads import rel_l2

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(__file__), "golden", "particle_state_00500_sub8.csv")


def _particle():
    p = read_particle_state(FIX)
    return p, Particle(x=p["x"], y=p["y"], s=p["s"], vorticity=p["vorticity"], isActive=p["active"])


def test_plain_velocity_matches_oracle(ctx, port):
    p, part = _particle()
    VelocityCalc(ctx, default_params(), u_inf=1.0, v_inf=0.0).get_velocity(part)
    q = -p["vorticity"] * p["s"] ** 2 / (2 * np.pi)
    ex, ey = port.fmm2d_field(p["x"], p["y"], q, p["active"])
    assert rel_l2((part.u, part.v), (ey + 1.0, -ex)) <= 1e-10


def test_mixed_velocity_matches_direct_sum(ctx, port):
    p, part = _particle()
    VelocityCalc(ctx, default_params(precision=PREC_MIXED)).get_velocity(part)
    q = -p["vorticity"] * p["s"] ** 2 / (2 * np.pi)
    tg = np.arange(p["x"].size)
    dx, dy = port.direct2d_field(p["x"], p["y"], q, p["active"], tg)
    assert rel_l2((part.u, part.v), (dy, -dx)) <= 1e-4
