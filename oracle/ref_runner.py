"""Runs the reference program built from its own sources (oracle/_ref) and
reads back its FP64 state dumps.

TEST INFRASTRUCTURE ONLY.  Only tests, fixture generation, `smoke()` and the
CPU-baseline legs of bench.py may use this module; the product never does.

The binaries are produced by oracle/ref_build/Makefile from the unmodified
reference sources.  A run is described by a UDF key file
(kapsel3_b200.udf.write_udf_keys); the dump format is written by
oracle/ref_build/ref_dump.cxx:
  header  int32[8]: magic 0x4b53504d, version 1, NX, NY, NZ, NZ_, Np, fields_every
  frame   int32[2]: ts, has_fields
          f64[5]:   time, degree_oblique, uk_dc[3]
          has_fields>=1: zeta0, zeta1, phi (each NX*NY*NZ_ f64, reference layout)
          has_fields==2: u (3 real fields, padded rows; Navier_Stokes runs)
          has_fields==10+N_spec: u, then N_spec k-space concentration fields
                      (Electrolyte runs)
          f64[Np*44]: per particle x, x_nopbc, v, v_old, omega, omega_old,
                      q(s,v), q_old(s,v), f_hydro, f_hydro_previous,
                      torque_hydro, torque_hydro_previous, fr, fr_previous
"""
from __future__ import annotations

import os
import subprocess
import tempfile
from typing import Dict, List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# The reference source tree: the environment variable KAPSEL_REFERENCE_TREE,
# else the tree the build of REF_DIR recorded in REF_DIR/REFERENCE_TREE.
TREE_RECORD = os.path.join(REF_DIR, "REFERENCE_TREE")


def reference_tree() -> Optional[str]:
    p = os.environ.get("KAPSEL_REFERENCE_TREE")
    if not p and os.path.exists(TREE_RECORD):
        p = open(TREE_RECORD).read().strip()
    return p if p and os.path.isdir(p) else None
PARTICLE_FIELDS = [("x", 3), ("x_nopbc", 3), ("v", 3), ("v_old", 3), ("omega", 3), ("omega_old", 3),
                   ("q", 4), ("q_old", 4), ("f_hydro", 3), ("f_hydro_previous", 3),
                   ("torque_hydro", 3), ("torque_hydro_previous", 3), ("fr", 3), ("fr_previous", 3)]
PARTICLE_WORDS = sum(n for _, n in PARTICLE_FIELDS)


def ref_binary(omp: bool = False, gpu_shim: bool = False, gpu_resident: bool = False) -> Optional[str]:
    """kapsel_ref (serial), kapsel_ref_omp (OpenMP), kapsel_gpu (serial, with
    the reference's boundary functions linked to the B200 library through
    kapsel3_b200/shim) or kapsel_gpu_resident (OpenMP host part, its main loop
    advanced on the GPU by kapsel3_b200/shim/kapsel_b200_resident.cxx)."""
    name = ("kapsel_gpu_resident" if gpu_resident else "kapsel_gpu" if gpu_shim
            else ("kapsel_ref_omp" if omp else "kapsel_ref"))
    p = os.path.join(REF_DIR, name)
    return p if os.access(p, os.X_OK) else None


def available(omp: bool = False, gpu_shim: bool = False, gpu_resident: bool = False) -> bool:
    return ref_binary(omp, gpu_shim, gpu_resident) is not None


def run_reference(keys_path: str, dump_path: Optional[str] = None, fields_every: int = 1,
                  body_force=(0.0, 0.0, 0.0), omp: bool = False, threads: Optional[int] = None,
                  step_times_path: Optional[str] = None, timeout: float = 3600.0, gpu_shim: bool = False,
                  gpu_resident: bool = False, restart_path: Optional[str] = None,
                  out_udf_path: Optional[str] = None) -> str:
    """Runs the reference program on a key file; with restart_path, its
    restart file (written at the end of every run, Save_Restart_udf) goes
    there as a key file that a later run can take as its input; with
    out_udf_path, its output UDF (the Output_udf records of a run with
    output.UDF = ON) goes there as record[n].<path> key lines."""
    exe = ref_binary(omp, gpu_shim, gpu_resident)
    if exe is None:
        raise FileNotFoundError("oracle/_ref is not built (make -C oracle/ref_build)")
    env = dict(os.environ)
    if dump_path:
        env["KAPSEL_REF_DUMP"] = dump_path
        env["KAPSEL_REF_FIELDS_EVERY"] = str(fields_every)
    if any(f != 0.0 for f in body_force):
        env["KAPSEL_REF_BODY_FORCE"] = ",".join(repr(float(f)) for f in body_force)
    if step_times_path:
        env["KAPSEL_REF_STEP_TIMES"] = step_times_path
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    wd = tempfile.mkdtemp(prefix="kapsel_ref_")
    cmd = [exe, f"-I{keys_path}", f"-O{out_udf_path or wd + '/out.udf'}", f"-D{wd}/def.udf",
           f"-R{restart_path or wd + '/res.udf'}"]
    open(f"{wd}/def.udf", "w").close()
    r = subprocess.run(cmd, env=env, cwd=wd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stderr[-3000:]}")
    return r.stderr


def run_reference_avs(keys_path: str, timeout: float = 600.0) -> str:
    """Runs kapsel_ref_avs (the serial reference with its own legacy AVS
    output) on a key file; the files go to the key file's
    output.ON.Out_dir."""
    exe = os.path.join(REF_DIR, "kapsel_ref_avs")
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError("oracle/_ref/kapsel_ref_avs is not built (make -C oracle/ref_build)")
    wd = tempfile.mkdtemp(prefix="kapsel_ref_avs_")
    open(f"{wd}/def.udf", "w").close()
    cmd = [exe, f"-I{keys_path}", f"-O{wd}/out.udf", f"-D{wd}/def.udf", f"-R{wd}/res.udf"]
    r = subprocess.run(cmd, cwd=wd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference run failed ({r.returncode}):\n{r.stderr[-3000:]}")
    return r.stderr


def read_dump(path: str) -> Dict:
    raw = open(path, "rb").read()
    hdr = np.frombuffer(raw, dtype=np.int32, count=8)
    if hdr[0] != 0x4B53504D:
        raise ValueError("not a reference dump")
    nx, ny, nz, nz_, npart, _ = (int(v) for v in hdr[2:8])
    nfield = nx * ny * nz_
    off = 32
    frames: List[Dict] = []
    while off < len(raw):
        ts, has_fields = np.frombuffer(raw, dtype=np.int32, count=2, offset=off)
        off += 8
        t, deg, u0, u1, u2 = np.frombuffer(raw, dtype=np.float64, count=5, offset=off)
        off += 40
        fr: Dict = dict(ts=int(ts), time=float(t), degree_oblique=float(deg),
                        uk_dc=np.array([u0, u1, u2]))
        if has_fields:
            def take(n):
                nonlocal off
                a = np.frombuffer(raw, dtype=np.float64, count=n, offset=off).copy()
                off += 8 * n
                return a
            z0 = take(nfield).reshape(nx, ny, nz_)
            z1 = take(nfield).reshape(nx, ny, nz_)
            fr["zeta"] = np.stack([z0, z1]).view(np.complex128)  # [2, NX, NY, NZ/2+1]
            fr["phi"] = take(nfield).reshape(nx, ny, nz_)[:, :, :nz].copy()
            if has_fields == 2 or has_fields >= 10:
                fr["u"] = take(3 * nfield).reshape(3, nx, ny, nz_)[..., :nz].copy()
            if has_fields >= 10:  # Electrolyte: k-space concentration of each ion species
                ns = has_fields - 10
                fr["conc"] = take(ns * nfield).reshape(ns, nx, ny, nz_).view(np.complex128)
        prec = np.frombuffer(raw, dtype=np.float64, count=npart * PARTICLE_WORDS, offset=off)
        off += 8 * npart * PARTICLE_WORDS
        prec = prec.reshape(npart, PARTICLE_WORDS)
        c = 0
        for name, n in PARTICLE_FIELDS:
            fr[name] = prec[:, c:c + n].copy()
            c += n
        frames.append(fr)
    return dict(shape=(nx, ny, nz), n_particles=npart, frames=frames)
