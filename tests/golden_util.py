"""Loading of the golden fixtures written by tests/golden/make_golden.py."""
import glob
import json
import os

import numpy as np

from kapsel3_b200.udf import SPMConfig

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# columns of the reference's Lees-Edwards stress line (sp_3d_ns.h:325-339)
STRESS_KEYS = ("time", "shear_rate", "degree_oblique", "strain", "lj", "hydro_old", "hydro_new", "reynolds", "fluid")


def fixture_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def _config(name):
    return json.loads(str(np.load(os.path.join(GOLDEN, name + ".npz"))["config_json"]))


def small_fixture_names(max_points=64 ** 3):
    """Fixtures of spherical particles on grids the numpy oracle steps in
    well under a second (the oracle has no rigid bodies)."""
    out = []
    for n in fixture_names():
        c = _config(n)
        if (1 << c["npx"]) * (1 << c["npy"]) * (1 << c["npz"]) <= max_points and not c.get("rigid"):
            out.append(n)
    return out


def rigid_fixture_names():
    return [n for n in fixture_names() if _config(n).get("rigid")]


def load(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    c = json.loads(str(z["config_json"]))
    c["fix_cell"] = tuple(c["fix_cell"])
    c["body_force"] = tuple(c["body_force"])
    cfg = SPMConfig(**c)
    parts = dict(x=z["init_x"], v=z["init_v"], omega=z["init_omega"], q=z["init_q"])
    return cfg, parts, z


def retained(cfg, zeta):
    d = cfg.derived()
    nx, ny, nz = cfg.shape
    kx = np.arange(nx)
    kx = np.where(kx > nx // 2, kx - nx, kx)
    ky = np.arange(ny)
    ky = np.where(ky > ny // 2, ky - ny, ky)
    ix = np.where(np.abs(kx) < d["TRN_X"])[0]
    iy = np.where(np.abs(ky) < d["TRN_Y"])[0]
    return zeta[:, ix][:, :, iy][:, :, :, :d["TRN_Z"]]


def rel(a, b):
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / (nb if nb > 0 else 1.0))


def check_state(z, frame, cfg, x, v, omega, q, fh_prev, zeta=None, u=None, tol=1e-10, ts=None):
    """Compares one state against trajectory frame `frame` of a fixture (step
    ts, default ts = frame for fixtures that store every step); returns the
    worst relative error and a dict of all."""
    ts = frame if ts is None else ts
    i = frame
    errs = {"x": rel(x, z["traj_x"][i]), "v": rel(v, z["traj_v"][i]), "omega": rel(omega, z["traj_omega"][i]),
            "q": rel(q, z["traj_q"][i]), "f_hydro": rel(fh_prev, z["traj_f_hydro_previous"][i])}
    if zeta is not None and f"zeta_retained_{ts}" in z.files:
        errs["zeta"] = rel(retained(cfg, zeta), z[f"zeta_retained_{ts}"])
    if u is not None and f"u_plane_{ts}" in z.files:
        errs["u_plane"] = rel(u[:, :, :, 0], z[f"u_plane_{ts}"])
        errs["u_sumsq"] = rel(np.array([np.sum(u[c] ** 2) for c in range(3)]), z[f"u_checksums_{ts}"][3:6])
    return max(errs.values()), errs
