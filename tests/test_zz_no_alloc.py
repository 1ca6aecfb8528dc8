"""The allocation-free entry point spm_make_f_particle_dt_sole_noalloc.

Some callers of this library cannot allocate device memory (their GPU memory
comes from their own pool or from another runtime, or their time loop must
not call the allocator).  This entry point serves them: the caller passes
device buffers for inputs and outputs and the call uses only a fixed device
array built into the library.  The test calls it through the C ABI twice in
a row, with different inputs, on the smallest grid (8 points per axis), a
ragged one and the largest (64^3, whose three fields fill the fixed array),
and compares each result with the existing context-based entry point
spm_make_f_particle_dt_sole_host and with the oracle's Solenoidal_u of
up - min(phi, 1) u (FP64, 1e-11 relative).  It is collected last so that a
run stopping at the first failure has already run every other test, and it
works in a fresh process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from kapsel3_b200 import _native as N
from kapsel3_b200.spm import SPMRun
from kapsel3_b200.udf import SPMConfig
from oracle.spm_oracle import OracleSPM

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _inputs(cfg, seed):
    rng = np.random.default_rng(seed)
    u = rng.standard_normal((3,) + cfg.shape)
    up = rng.standard_normal((3,) + cfg.shape)
    phi = np.clip(rng.random(cfg.shape) * 1.3, 0.0, 1.0)
    return u, up, phi


def _no_particles():
    z = np.zeros((0, 3))
    return {"x": z, "v": z, "omega": z, "q": np.zeros((0, 4))}


@pytest.mark.parametrize("np3", [(3, 3, 3), (5, 4, 6), (6, 6, 6)])
def test_noalloc_matches_context_entry_point_and_oracle(gpu, np3):
    import torch

    cfg = SPMConfig(npx=np3[0], npy=np3[1], npz=np3[2], n_particles=0, lj_truncate="NONE")
    nx, ny, nz = cfg.shape
    nzp = 2 * (nz // 2 + 1)
    L = N.lib()
    oracle = OracleSPM(cfg, _no_particles())
    with SPMRun(cfg) as run:
        for call, seed in enumerate((101, 202)):
            u, up, phi = _inputs(cfg, seed + sum(np3))
            want = run.Make_f_particle_dt_sole(u, up, phi)
            ref = oracle.solenoidal_u(up - np.minimum(phi, 1.0) * u)

            def dev(a):
                padded = np.zeros((nx, ny, nzp))
                padded[:, :, :nz] = a
                return torch.from_numpy(padded).cuda()

            ud = [dev(u[d]) for d in range(3)]
            upd = [dev(up[d]) for d in range(3)]
            phid = dev(phi)
            fd = [torch.full((nx, ny, nzp), float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
            torch.cuda.synchronize()
            ptrs = [C.c_void_p(t.data_ptr()) for t in ud + upd + [phid] + fd]
            rc = L.spm_make_f_particle_dt_sole_noalloc(*ptrs, cfg.npx, cfg.npy, cfg.npz, None)
            assert rc == 0, L.spm_last_error()
            torch.cuda.synchronize()
            got = np.stack([t.cpu().numpy()[:, :, :nz] for t in fd])
            assert np.isfinite(got).all(), f"call {call}: output not fully written"
            assert _rel(got, want) < 1e-11, (call, _rel(got, want))
            assert _rel(got, ref) < 1e-11, (call, _rel(got, ref))


def test_noalloc_rejects_grids_beyond_its_scratch(gpu):
    L = N.lib()
    assert L.spm_make_f_particle_dt_sole_noalloc(*[C.c_void_p(8)] * 10, 7, 5, 5, None) == 1
    assert b"8..64" in L.spm_last_error()
    assert L.spm_make_f_particle_dt_sole_noalloc(*[C.c_void_p(8)] * 10, 5, 2, 5, None) == 1
