"""GPU pair models vs the reference's outputs (golden) and the FP64 oracle.

Tolerances:
  precision="fp64":  rtol 1e-9 against the reference FP64 torch path.
  precision="mixed": FP32 pair arithmetic -> relative force error
                     max|dF| / max|F| <= 1e-5 and |dE|/|E| <= 5e-6.
"""

import numpy as np
import pytest
import torch

from oracle import pair as opair

pytestmark = pytest.mark.gpu


def _state(c):
    from tsb.state import SimState

    dev = torch.device("cuda")
    return SimState(positions=torch.as_tensor(c["positions"], device=dev),
                    masses=torch.ones(len(c["positions"]), dtype=torch.float64, device=dev),
                    cell=torch.as_tensor(c["cell"], device=dev),
                    pbc=torch.as_tensor(c["pbc"], dtype=torch.bool, device=dev),
                    atomic_numbers=torch.as_tensor(c["atomic_numbers"], device=dev),
                    system_idx=torch.as_tensor(c["system_idx"], dtype=torch.int64, device=dev))


def _make(key, precision):
    from tsb import models

    kw = dict(compute_stress=True, per_atom_energies=True, per_atom_stresses=True,
              precision=precision)
    if key == "lj_ar":
        return models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405, **kw)
    if key == "lj_shifted":
        return models.LennardJonesModel(sigma=3.405, epsilon=0.0104, cutoff=2.5 * 3.405,
                                        shift_energy=True, **kw)
    if key == "morse_cu":
        return models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, **kw)
    if key == "morse_slab":
        return models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=5.0, **kw)
    if key == "soft_sphere":
        return models.SoftSphereModel(sigma=2.6, epsilon=0.05, alpha=2.0, **kw)
    if key == "soft_sphere_a3":
        return models.SoftSphereModel(sigma=2.6, epsilon=0.05, alpha=3.5, **kw)
    if key.startswith("soft_sphere_multi"):
        alp = [[2.0, 3.0], [3.0, 2.0]] if key.endswith("int") else [[2.0, 2.5], [2.5, 3.0]]
        return models.SoftSphereMultiModel(
            atomic_numbers=torch.tensor([18, 36]),
            sigma_matrix=torch.tensor([[2.6, 2.9], [2.9, 3.1]], dtype=torch.float64),
            epsilon_matrix=torch.tensor([[0.05, 0.07], [0.07, 0.04]], dtype=torch.float64),
            alpha_matrix=torch.tensor(alp, dtype=torch.float64), **kw)
    if key == "ka_lj":
        return models.kob_andersen_model(**kw)
    raise KeyError(key)


CASES = ["lj_ar", "lj_shifted", "morse_cu", "morse_slab", "soft_sphere", "soft_sphere_a3",
         "soft_sphere_multi", "soft_sphere_multi_int", "ka_lj"]
KEYS = ("energy", "forces", "stress", "energies", "stresses")


@pytest.mark.parametrize("case", CASES)
def test_models_fp64_match_reference(golden, case):
    c = golden["models"][case]
    out = _make(case, "fp64")(_state(c))
    for k in KEYS:
        got = out[k].cpu().numpy()
        ref = c[k]
        ok = np.isfinite(ref)  # reference NaN artefact, see test_oracle_golden
        np.testing.assert_allclose(got[ok], ref[ok], rtol=1e-9, atol=1e-12, err_msg=k)
        assert np.isfinite(got).all()


@pytest.mark.parametrize("case", CASES)
def test_models_mixed_precision_error(golden, case):
    c = golden["models"][case]
    out = _make(case, "mixed")(_state(c))
    ref = _make(case, "fp64")(_state(c))
    f, fr = out["forces"].cpu().numpy(), ref["forces"].cpu().numpy()
    err = np.abs(f - fr).max() / np.abs(fr).max()
    assert err <= 1e-5, err
    # energy: FP32 r^2 feeds (sigma/r)^12, so the pair energy carries ~6x the FP32
    # rounding of r^2 (KA random starts overlap: E ~ 1e9 eV); sums are FP64
    e, er = out["energy"].cpu().numpy(), ref["energy"].cpu().numpy()
    assert np.all(np.abs(e - er) <= 5e-6 * np.abs(er) + 1e-9)
    s, sr = out["stress"].cpu().numpy(), ref["stress"].cpu().numpy()
    assert np.abs(s - sr).max() <= 1e-5 * np.abs(sr).max() + 1e-12


def test_model_float32_state(golden):
    from tsb import models
    from tsb.state import SimState

    c = golden["models"]["morse_cu"]
    st = _state(c)
    st32 = SimState(positions=st.positions.float(), masses=st.masses.float(),
                    cell=st.cell.float(), pbc=st.pbc, atomic_numbers=st.atomic_numbers,
                    system_idx=st.system_idx)
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          dtype=torch.float32, compute_stress=True)
    out = m(st32)
    assert out["forces"].dtype == torch.float32
    err = np.abs(out["forces"].cpu().numpy() - c["forces"]).max() / np.abs(c["forces"]).max()
    assert err < 1e-4
    with pytest.raises(TypeError):
        models.MorseModel(dtype=torch.float64)(st32)


def test_model_properties_sum_forces_stress_symmetry(golden):
    """Sum of forces 0, symmetric stress (test_pair_potential.py:231-252)."""
    c = golden["models"]["morse_cu"]
    out = _make("morse_cu", "fp64")(_state(c))
    f = out["forces"].cpu().numpy()
    sysi = c["system_idx"]
    for s in np.unique(sysi):
        assert np.abs(f[sysi == s].sum(0)).max() < 1e-10
    st = out["stress"].cpu().numpy()
    np.testing.assert_allclose(st, np.transpose(st, (0, 2, 1)), atol=1e-12)


def test_model_wrapped_vs_unwrapped_positions(golden):
    """Energies/forces invariant to integer lattice translations of atoms
    (test_pair_potential.py:273-303)."""
    c = dict(golden["models"]["morse_cu"])
    rng = np.random.default_rng(0)
    cell_row = np.transpose(c["cell"], (0, 2, 1))
    shifts = rng.integers(-3, 4, size=(len(c["positions"]), 3)).astype(float)
    c2 = dict(c)
    c2["positions"] = c["positions"] + np.einsum("nk,nkm->nm", shifts,
                                                 cell_row[c["system_idx"]])
    m = _make("morse_cu", "fp64")
    a, b = m(_state(c)), m(_state(c2))
    np.testing.assert_allclose(a["forces"].cpu(), b["forces"].cpu(), atol=1e-10)
    np.testing.assert_allclose(a["energy"].cpu(), b["energy"].cpu(), rtol=1e-12)


def test_batched_equals_single(golden):
    """A system's result does not depend on the batch it is in."""
    c = golden["models"]["morse_cu"]
    m = _make("morse_cu", "mixed")
    full = m(_state(c))
    sysi = c["system_idx"]
    for s in (0, 3):
        sel = sysi == s
        cs = {"positions": c["positions"][sel], "cell": c["cell"][s:s + 1], "pbc": c["pbc"],
              "atomic_numbers": c["atomic_numbers"][sel],
              "system_idx": np.zeros(sel.sum(), dtype=np.int64)}
        one = m(_state(cs))
        assert torch.equal(one["forces"], full["forces"][torch.as_tensor(sel).cuda()])
        assert torch.equal(one["energy"][0], full["energy"][s])


def test_model_vs_oracle_random_boxes():
    from tsb import workloads

    d = workloads.kob_andersen_batch(5, 64, 400, seed=4)
    d["positions"] = d["positions"] + 0.0
    c = {**d}
    m = _make("ka_lj", "fp64")
    out = m(_state(c))
    o = opair.pair_forward(opair.LJ, opair.kob_andersen_table(), d["atomic_numbers"] - 1,
                           d["positions"], np.transpose(d["cell"], (0, 2, 1)), d["pbc"],
                           d["system_idx"], 2.5 * 3.4)
    np.testing.assert_allclose(out["forces"].cpu().numpy(), o["forces"], rtol=1e-9,
                               atol=1e-9 * np.abs(o["forces"]).max())
    np.testing.assert_allclose(out["energy"].cpu().numpy(), o["energy"], rtol=1e-9)
