"""The oracle (numpy restatement) against the fixtures produced by the
reference program itself (tests/golden/make_golden.py): pins the oracle on
any machine, with or without the reference sources."""
import numpy as np
import pytest

from kapsel3_b200.udf import EQ_LE
from oracle.spm_oracle import OracleSPM, OracleSPMLE
from tests.golden_util import STRESS_KEYS, check_state, fixture_names, load, rigid_fixture_names, small_fixture_names

TOL = 1e-12


# The 128^3 fixture is checked against the GPU FP64 path only: the numpy
# oracle would need minutes per hundred steps there.
@pytest.mark.parametrize("name", small_fixture_names())
def test_oracle_matches_reference_fixture(name):
    cfg, parts, z = load(name)
    le = cfg.equation == EQ_LE
    o = (OracleSPMLE if le else OracleSPM)(cfg, parts)
    nframes = len(z["traj_ts"])
    steps = set(int(s) for s in z["field_steps"])
    for ts in range(nframes):
        want_fields = ts in steps
        u = o.velocity_field() if (want_fields and not le) else None
        worst, errs = check_state(z, ts, cfg, o.x, o.v, o.omega, o.q, o.f_hydro_previous,
                                  zeta=o.zeta if want_fields else None, u=u)
        assert worst < TOL, (name, ts, errs)
        if le:
            assert abs(o.gamma - z["traj_degree_oblique"][ts]) < 1e-14
        if ts + 1 < nframes:
            o.step()
            if le:
                # the reference prints 8 significant digits
                ref = z["stress_lines"][ts]
                for i, k in enumerate(STRESS_KEYS):
                    assert abs(o.stress[k] - ref[i]) <= 6e-8 * abs(ref[i]) + 1e-20, (name, ts, k, o.stress[k], ref[i])


def test_fixtures_present():
    assert len(fixture_names()) >= 3


@pytest.mark.parametrize("name", rigid_fixture_names())
def test_rigid_fixture_invariants(name):
    """Rigid-body fixtures (no oracle restatement; the GPU path is compared
    with them directly): every body keeps its shape, its beads share one
    orientation and one angular velocity (update_Particle_Configuration,
    rigid.h:171-188; set_Particle_Velocities, rigid.h:213-225)."""
    cfg, parts, z = load(name)
    first = [0]
    for beads, count, *_ in cfg.rigid:
        for _ in range(int(count)):
            first.append(first[-1] + int(beads))
    assert first[-1] == cfg.n_particles == z["traj_x"].shape[1]
    xs, ws, qs = z["traj_x_nopbc"], z["traj_omega"], z["traj_q"]
    for b in range(len(first) - 1):
        sl = slice(first[b], first[b + 1])
        d0 = np.linalg.norm(xs[0, sl, None, :] - xs[0, None, sl, :], axis=-1)
        for t in range(len(z["traj_ts"])):
            x, w, q = xs[t, sl], ws[t, sl], qs[t, sl]
            assert (q == q[0]).all() and (w == w[0]).all(), (name, t, b)
            assert abs(np.linalg.norm(q[0]) - 1.0) < 1e-13
            d = np.linalg.norm(x[:, None, :] - x[None, :, :], axis=-1)
            assert np.abs(d - d0).max() < 1e-11, (name, t, b)
