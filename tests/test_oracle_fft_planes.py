"""The oracle's inverse transform against the reference's own (A_k2a with
Ooura's rdft3dsort + rdft3d, fft_wrapper.h:662-681, fftsg3d.c:632-655),
built from the reference sources into oracle/_ref/ooura_inverse: on
Hermitian spectra, on gradients i k a (not Hermitian on the Nyquist
wavenumbers, the Coulomb force path of the Electrolyte step) and on spectra
with every entry random."""
import os
import subprocess

import numpy as np
import pytest

from oracle.spm_oracle import ooura_packed_planes

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "..", "oracle", "_ref", "ooura_inverse")

pytestmark = pytest.mark.skipif(not os.path.exists(BIN), reason="oracle/_ref/ooura_inverse is not built")


def reference_inverse(ak, tmp_path):
    nx, ny, hz = ak.shape
    nz = 2 * (hz - 1)
    src, dst = str(tmp_path / "k.bin"), str(tmp_path / "r.bin")
    np.ascontiguousarray(ak, dtype=np.complex128).tofile(src)
    subprocess.run([BIN, str(nx), str(ny), str(nz), src, dst], check=True, timeout=60)
    return np.fromfile(dst).reshape(nx, ny, nz + 2)[:, :, :nz]


def oracle_inverse(ak):
    nx, ny, hz = ak.shape
    return np.fft.irfftn(ooura_packed_planes(ak), s=(nx, ny, 2 * (hz - 1)), axes=(0, 1, 2))


@pytest.mark.parametrize("shape", [(8, 4, 16), (4, 8, 8), (16, 16, 4)])
def test_packed_planes_match_the_reference_inverse(shape, tmp_path):
    nx, ny, nz = shape
    rng = np.random.default_rng(nx * 100 + ny * 10 + nz)
    a = rng.standard_normal(shape)
    A = np.fft.rfftn(a)
    kx = np.array([i - nx if i > nx // 2 else i for i in range(nx)])[:, None, None]
    ky = np.array([j - ny if j > ny // 2 else j for j in range(ny)])[None, :, None]
    kz = np.arange(nz // 2 + 1)[None, None, :]
    fields = {"hermitian": A, "d/dx": 1j * kx * A, "d/dy": 1j * ky * A, "d/dz": 1j * kz * A,
              "random": rng.standard_normal(A.shape) + 1j * rng.standard_normal(A.shape)}
    for name, F in fields.items():
        F = np.broadcast_to(F, A.shape)
        ref = reference_inverse(F, tmp_path)
        got = oracle_inverse(F)
        scale = max(np.abs(ref).max(), 1.0)
        assert np.abs(got - ref).max() <= 1e-13 * scale, (shape, name)
    # irfftn without the packed-plane rule differs on a Nyquist gradient
    D = 1j * kz * A
    assert np.abs(np.fft.irfftn(D, s=shape, axes=(0, 1, 2)) - reference_inverse(D, tmp_path)).max() > 1e-3
