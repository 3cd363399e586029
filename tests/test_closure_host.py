"""Host-side pieces of the learned closure's training data (no GPU): the
spectral-cutoff stresses and the FFT helpers they are built from."""
import numpy as np

from diablo_b200 import closure, layout, params as P


def _state(p, rng, les_only_of=None):
    """Random dealiased velocity spectra with a real (Hermitian) kx = 0 column;
    with les_only_of = q, only the modes q's grid keeps."""
    cu = []
    for _ in range(3):
        a = layout.new_fourier(p)
        blk = layout.dealiased(p, a)
        blk[...] = rng.standard_normal(blk.shape) + 1j * rng.standard_normal(blk.shape)
        blk[:, :, 0] = 0.0
        if les_only_of is not None:
            keep = np.zeros(blk.shape[1:], dtype=bool)
            keep[np.ix_(closure._les_kz(p, les_only_of.nz // 3), np.arange(les_only_of.nx // 3 + 1))] = True
            blk[:, ~keep] = 0.0
        cu.append(a)
    return {"cu": cu}


def test_fourier_round_trip_on_kept_modes():
    rng = np.random.default_rng(1)
    f = rng.standard_normal((4, 32, 48))
    spec = closure._to_fourier(f, 10, 12)
    again = closure._to_fourier(closure._to_physical(spec, 48, 32), 10, 12)
    assert np.abs(again - spec).max() < 1e-14


def test_to_physical_is_the_plain_mode_sum():
    # one mode kx = 2, kz = -3 with coefficient c: c e^{i(2x - 3z)} + conj
    spec = np.zeros((1, 2 * 4 + 1, 5), dtype=np.complex128)
    c = 0.3 - 0.7j
    spec[0, 2 * 4 + 1 - 3, 2] = c
    f = closure._to_physical(spec, 16, 12)
    z = np.arange(12)[:, None] * 2 * np.pi / 12
    x = np.arange(16)[None, :] * 2 * np.pi / 16
    want = 2 * np.real(c * np.exp(1j * (2 * x - 3 * z)))
    assert np.abs(f[0] - want).max() < 1e-13


def test_cutoff_stresses_vanish_for_a_resolved_field():
    p = P.kelvin_helmholtz(96, 65, 96)
    q = p.copy()
    q.nx, q.nz = 32, 32
    rng = np.random.default_rng(2)
    tau = closure.cutoff_stresses(p, q, _state(p, rng, les_only_of=q))
    full = closure.cutoff_stresses(p, q, _state(p, rng))
    assert tau.shape == (p.ny - 2, q.nz, q.nx, 6)
    assert np.abs(tau).max() < 1e-9 * np.abs(full).max()
    assert np.abs(full).max() > 1.0
