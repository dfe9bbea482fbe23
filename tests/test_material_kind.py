"""The native material classifier (emg_material_classify, host threads)
against numpy's definition of the same checks, on edge cases: isotropic,
diagonal, full, identity, NaN on and off the diagonal, -0.0 off the
diagonal, an almost-identity. Host-only: no GPU is used."""
import numpy as np
import pytest

from emerge_b200.assembly import _is_identity, classify_material, material_kind


def _cases():
    rng = np.random.default_rng(0)
    nT = 200_003  # several host threads, a ragged last range
    v = rng.normal(size=nT) + 1j * rng.normal(size=nT)
    iso = np.zeros((3, 3, nT), complex)
    for d in range(3):
        iso[d, d] = v
    ident = np.zeros((3, 3, nT), complex)
    for d in range(3):
        ident[d, d] = 1
    out = {"iso": iso, "identity": ident}
    t = iso.copy(); t[1, 1, 5] += 1.0; out["diag"] = t
    t = iso.copy(); t[2, 0, nT - 1] = 1e-300j; out["full_last"] = t
    t = iso.copy(); t[0, 1, 0] = 2.0; out["full_first"] = t
    t = iso.copy(); t[0, 0, 7] = np.nan; out["nan_diag"] = t
    t = ident.copy(); t[1, 2, 3] = np.nan; out["nan_off"] = t
    t = ident.copy(); t[0, 1] = -0.0; out["neg_zero_off"] = t
    t = ident.copy(); t[2, 2, 9] = 1 + 1e-16j; out["almost_identity"] = t
    out["empty"] = np.zeros((3, 3, 0), complex)
    out["tiny"] = ident[:, :, :3].copy()
    return out


@pytest.mark.parametrize("name", list(_cases()))
def test_native_classifier_matches_numpy(name):
    t = _cases()[name]
    assert material_kind(t) == (classify_material(t), _is_identity(t))


def test_real_and_complex64_inputs_are_converted():
    t = np.zeros((3, 3, 1000), np.float32)
    for d in range(3):
        t[d, d] = 2.0
    assert material_kind(t) == (classify_material(t.astype(complex)), False)
