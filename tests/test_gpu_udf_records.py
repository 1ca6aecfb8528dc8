"""Per-frame UDF particle records (spm_udf_out_open / _record / _close)
against the records the reference program writes itself with output.UDF =
ON (Output_udf, output.cxx:268-375; through the UDF stand-in of
oracle/ref_build, as record[n].<path> key lines): the same keys in every
record, t equal, and every value within 1e-9 relative (the FP64 states of
the two programs differ by ~1e-12 after a few steps).  Covered: spheres
with the thermostat, rigid bodies under gravity (beads' positions as centre
+ offset without a wrap, the RigidParticles[] records) and squirmers (the
slip force and torque of the previous step)."""
import os

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import SPMConfig, make_particles, make_rigid_bodies, read_udf_keys, write_udf_keys
from oracle import ref_runner

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_runner.available(), reason="reference program not built (oracle/_ref)")]

CASES = {
    "spheres_thermostat": SPMConfig(npx=5, npy=5, npz=5, n_particles=3, a=3.5, a_xi=2.0, dt=0.05, kbt=1e-4,
                                    gts=2, num_snap=3),
    "rigid_gravity": SPMConfig(npx=5, npy=5, npz=5, n_particles=6, a=3.0, a_xi=2.0, dt=0.05, gts=2, num_snap=3,
                               rigid=((3, 2, 1.5, "free", (0.0, 0.0, 0.0), (0.0, 0.0, 0.0)),),
                               rigid_gravity=(0.0, 1e-3, 0.0)),
    "squirmers": SPMConfig(npx=5, npy=5, npz=5, n_particles=2, a=4.0, a_xi=2.0, dt=0.1, gts=2, num_snap=2,
                           janus_axis="Z", janus_propulsion="SQUIRMER", slip_vel=0.015, slip_mode=2.0,
                           slip_tol=0.005, slip_iter=4),
}


def _records(path):
    out = {}
    for k, v in read_udf_keys(path).items():
        n, key = k.split("].", 1)
        out.setdefault(int(n[len("record["):]), {})[key] = v
    return [out[i] for i in sorted(out)]


@pytest.mark.parametrize("name", sorted(CASES))
def test_udf_records_match_the_reference_program(gpu, name, tmp_path):
    cfg = CASES[name]
    if cfg.rigid:
        parts = make_rigid_bodies(cfg, seed=6, straddle=True)
    else:
        parts = make_particles(cfg, seed=6, v_sd=1e-3, random_orientation=True)
    keys = str(tmp_path / "in.keys")
    write_udf_keys(keys, cfg, parts, out_dir=str(tmp_path / "avs"))
    kv = read_udf_keys(keys)
    kv["output.UDF"] = "ON"
    with open(keys, "w") as f:
        f.writelines(f"{k} = {v}\n" for k, v in kv.items())
    ref_path = str(tmp_path / "ref_out.keys")
    ref_runner.run_reference(keys, out_udf_path=ref_path)
    ours_path = str(tmp_path / "gpu_out.keys")
    with SPMRun(cfg) as run:
        run.initialize(parts)
        run.udf_out_open(ours_path)
        for ts in range(cfg.mstep + 1):  # a record at every frame, then the step
            if ts % cfg.gts == 0:
                run.udf_out_record()
            run.step(1)
        run.udf_out_close()
    ref, ours = _records(ref_path), _records(ours_path)
    assert len(ref) == len(ours) == cfg.num_snap + 1
    for n, (a, b) in enumerate(zip(ours, ref)):
        assert set(a) == set(b), (n, sorted(set(a) ^ set(b))[:8])
        assert int(a["t"]) == int(b["t"]) == n * cfg.gts
        # each value against the largest magnitude of its field in the record
        scale = {}
        for k, v in b.items():
            field = k.split("].")[-1]
            scale[field] = max(scale.get(field, 0.0), abs(float(v)))
        for k in b:
            tol = 1e-9 * scale[k.split("].")[-1]]
            assert abs(float(a[k]) - float(b[k])) <= tol, (name, n, k, a[k], b[k])


def test_udf_record_without_open_is_refused(gpu):
    cfg = CASES["spheres_thermostat"]
    with SPMRun(cfg) as run:
        run.initialize(make_particles(cfg, seed=1))
        with pytest.raises(N.SpmError, match="spm_udf_out_open was not called"):
            run.udf_out_record()
