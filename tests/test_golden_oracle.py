"""The oracle (numpy restatement) against the fixtures produced by the
reference program itself (tests/golden/make_golden.py): pins the oracle on
any machine, with or without the reference sources."""
import numpy as np
import pytest

from oracle.spm_oracle import OracleSPM
from tests.golden_util import check_state, fixture_names, load

TOL = 1e-12


@pytest.mark.parametrize("name", fixture_names())
def test_oracle_matches_reference_fixture(name):
    cfg, parts, z = load(name)
    o = OracleSPM(cfg, parts)
    nframes = len(z["traj_ts"])
    steps = set(int(s) for s in z["field_steps"])
    for ts in range(nframes):
        want_fields = ts in steps
        u = o.velocity_field() if want_fields else None
        worst, errs = check_state(z, ts, cfg, o.x, o.v, o.omega, o.q, o.f_hydro_previous,
                                  zeta=o.zeta if want_fields else None, u=u)
        assert worst < TOL, (name, ts, errs)
        if ts + 1 < nframes:
            o.step()


def test_fixtures_present():
    assert len(fixture_names()) >= 3
