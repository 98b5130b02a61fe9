"""Pin the CPU oracle against golden vectors produced by the reference itself."""

import numpy as np
import pytest

from oracle import fire as ofire
from oracle import linalg3, md as omd, neighbors as onl, pair as opair

NL_CASES = ["ar_fcc444", "cu_tri_batch", "slab_pbc_TTF", "cluster_nopbc",
            "tiny_self_images", "rhombohedral_unwrapped"]


def _golden_set(g, key):
    m, sm, sh = g[key]["mapping"], g[key]["system_mapping"], g[key]["shifts"]
    return onl.sort_pairs(m, sm, sh)


@pytest.mark.parametrize("case", NL_CASES)
@pytest.mark.parametrize("self_interaction", [False, True])
def test_nl_oracle_matches_reference(golden, case, self_interaction):
    g = golden["nl"]
    c = g[case]
    key = case + ("_self" if self_interaction else "")
    ref = _golden_set(g, key)
    got = onl.neighbor_list(c["positions"], c["cell_row"], c["pbc"], float(c["cutoff"]),
                            c["system_idx"].astype(np.int64), self_interaction)
    assert got[0].shape == ref[0].shape
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(got[1], ref[1])
    assert np.array_equal(np.rint(got[2]).astype(int), ref[2].astype(int))
    # the reference's own two backends agree on the count (torch_nl_n2 cross-check)
    if case not in ("tiny_self_images",):
        assert int(g[key]["n2_count"]) == ref[0].shape[1]


def _model_case(golden, key):
    return golden["models"][key]


def _species(z, zs):
    lut = {int(v): k for k, v in enumerate(zs)}
    return np.array([lut[int(v)] for v in z])


MODEL_CASES = {
    "lj_ar": (opair.LJ, opair.single_table(opair.LJ, 3.405, 0.0104), 2.5 * 3.405, None),
    "morse_cu": (opair.MORSE, opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588),
                 6.0, None),
    "morse_slab": (opair.MORSE, opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588),
                   5.0, None),
    "soft_sphere": (opair.SOFT, opair.single_table(opair.SOFT, 2.6, 0.05, 2.0), 2.6, None),
    "soft_sphere_a3": (opair.SOFT, opair.single_table(opair.SOFT, 2.6, 0.05, 3.5), 2.6,
                       None),
    "lj_shifted": (opair.LJ, opair.single_table(
        opair.LJ, 3.405, 0.0104, eshift=opair.lj_shift(3.405, 0.0104, 2.5 * 3.405)),
        2.5 * 3.405, None),
}


def _multi_ss_table(alp=((2.0, 2.5), (2.5, 3.0))):
    sig = np.array([[2.6, 2.9], [2.9, 3.1]])
    eps = np.array([[0.05, 0.07], [0.07, 0.04]])
    alp = np.array(alp)
    tab = np.zeros((2, 2, 5))
    tab[..., 0], tab[..., 1], tab[..., 2], tab[..., 3] = sig, eps, alp, np.inf
    return tab


@pytest.mark.parametrize("key", list(MODEL_CASES) + ["soft_sphere_multi",
                                                     "soft_sphere_multi_int", "ka_lj"])
def test_pair_oracle_matches_reference(golden, key):
    c = _model_case(golden, key)
    if key.startswith("soft_sphere_multi"):
        alp = ((2.0, 3.0), (3.0, 2.0)) if key.endswith("int") else ((2.0, 2.5), (2.5, 3.0))
        kind, tab, rc = opair.SOFT, _multi_ss_table(alp), 3.1
        species = _species(c["atomic_numbers"], [18, 36])
    elif key == "ka_lj":
        kind, tab, rc = opair.LJ, opair.kob_andersen_table(), 2.5 * 3.4
        species = c["atomic_numbers"] - 1
    else:
        kind, tab, rc, _ = MODEL_CASES[key]
        species = np.zeros(len(c["positions"]), dtype=int)
    cell_row = np.transpose(c["cell"], (0, 2, 1))
    out = opair.pair_forward(kind, tab, species, c["positions"], cell_row, c["pbc"],
                             c["system_idx"].astype(np.int64), rc, per_atom=True)
    for k in ("energy", "forces", "stress", "energies", "stresses"):
        ref = c[k]
        if key == "soft_sphere_multi" and k in ("forces", "stress", "stresses"):
            # The reference differentiates (1 - r/sigma)^alpha with non-integer alpha
            # through torch.where for pairs sigma_ij <= r < cutoff; autograd gives
            # 0 * NaN = NaN there (soft_sphere.py:164-166 + pair_potential.py:420).
            # The oracle returns the finite force; compare where the reference is finite.
            ok = np.isfinite(ref)
            assert (~ok).any() and np.isfinite(out[k]).all()
            np.testing.assert_allclose(out[k][ok], ref[ok], rtol=1e-10, atol=1e-12)
            continue
        np.testing.assert_allclose(out[k], ref, rtol=1e-10, atol=1e-12, err_msg=k)


def _lj_force_fn(cell, system_idx, pbc=(True, True, True)):
    tab = opair.single_table(opair.LJ, 3.405, 0.0104)

    def fn(q):
        o = opair.pair_forward(opair.LJ, tab, np.zeros(len(q), int), q,
                               np.transpose(cell, (0, 2, 1)), np.array(pbc), system_idx,
                               2.5 * 3.405)
        return o["energy"], o["forces"]
    return fn


def test_nve_oracle_matches_reference(golden):
    g = golden["md"]["nve"]
    sysi = g["system_idx"].astype(np.int64)
    fn = _lj_force_fn(g["cell"], sysi)
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0],
          "masses": g["masses"], "forces": g["forces"][0], "energy": g["energy"][0]}
    for k in range(1, g["positions"].shape[0]):
        st = omd.nve_step(st, fn, float(g["dt"]))
        np.testing.assert_allclose(st["positions"], g["positions"][k], rtol=1e-12,
                                   atol=1e-12)
        np.testing.assert_allclose(st["momenta"], g["momenta"][k], rtol=1e-10,
                                   atol=1e-13)
        np.testing.assert_allclose(st["energy"], g["energy"][k], rtol=1e-11)


def test_langevin_oracle_matches_reference(golden):
    g = golden["md"]["nvt"]
    sysi = g["system_idx"].astype(np.int64)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(g["cell"], (0, 2, 1)), np.array([True] * 3),
                               sysi, 6.0)
        return o["energy"], o["forces"]

    st = {"positions": g["positions"][0], "momenta": g["momenta"][0],
          "masses": g["masses"], "forces": g["forces"][0], "energy": g["energy"][0]}
    for k in range(1, g["positions"].shape[0]):
        st = omd.nvt_langevin_step(st, fn, float(g["dt"]), float(g["kT"]),
                                   float(g["gamma"]), g["noise"][k - 1], sysi)
        np.testing.assert_allclose(st["positions"], g["positions"][k], rtol=1e-12,
                                   atol=1e-12)
        np.testing.assert_allclose(st["momenta"], g["momenta"][k], rtol=1e-9, atol=1e-12)


def _ka_model(cell_unused, system_idx, z):
    tab = opair.kob_andersen_table()

    def model(q, cell_col):
        o = opair.pair_forward(opair.LJ, tab, z - 1, q, np.transpose(cell_col, (0, 2, 1)),
                               np.array([True] * 3), system_idx, 2.5 * 3.4)
        return o["energy"], o["forces"], o["stress"]
    return model


def test_fire_frechet_oracle_matches_reference(golden):
    g = golden["fire"]["ase_frechet"]
    sysi = g["system_idx"].astype(np.int64)
    model = _ka_model(None, sysi, g["atomic_numbers"])
    st = {"positions": g["positions"][0], "cell": g["cell"][0], "masses": g["masses"],
          "system_idx": sysi}
    st = ofire.fire_init(st, model, cell_filter="frechet")
    for k in range(1, g["positions"].shape[0]):
        st = ofire.fire_step(st, model)
        for key in ("positions", "cell", "energy", "forces", "cell_forces",
                    "cell_positions", "velocities", "dt", "alpha"):
            np.testing.assert_allclose(st[key], g[key][k], rtol=1e-8, atol=1e-10,
                                       err_msg=f"step {k} {key}")
        np.testing.assert_array_equal(st["n_pos"], g["n_pos"][k])


def test_fire_vv_oracle_matches_reference(golden):
    g = golden["fire"]["vv"]
    sysi = g["system_idx"].astype(np.int64)
    model = _ka_model(None, sysi, g["atomic_numbers"])
    st = {"positions": g["positions"][0], "cell": g["cell"], "masses": g["masses"],
          "system_idx": sysi}
    st = ofire.fire_init(st, model)
    for k in range(1, g["positions"].shape[0]):
        st = ofire.fire_step(st, model, flavor="vv_fire")
        for key in ("positions", "energy", "forces", "velocities", "dt", "alpha"):
            np.testing.assert_allclose(st[key], g[key][k], rtol=1e-9, atol=1e-11,
                                       err_msg=f"step {k} {key}")


def test_math_oracle_matches_reference(golden):
    m = golden["math"][""] if "" in golden["math"] else None
    import os

    from conftest import GOLDEN
    m = np.load(os.path.join(GOLDEN, "math.npz"))
    R, L = linalg3.expm_frechet(m["A"], m["E"])
    np.testing.assert_allclose(R, m["expA"], rtol=1e-13, atol=1e-14)
    np.testing.assert_allclose(L, m["L"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(linalg3.expm(m["A"]), m["expm_torch"], rtol=1e-13,
                               atol=1e-14)
    np.testing.assert_allclose(linalg3.logm(m["T"]), m["logT"], rtol=1e-10, atol=1e-13)


def _morse_fn(cell, sysi):
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(cell, (0, 2, 1)), np.array([True] * 3), sysi, 6.0)
        return o["energy"], o["forces"]
    return fn


def test_nose_hoover_oracle_matches_reference(golden):
    from oracle import thermostats as oth

    s, g = golden["thermostats"]["sys"], golden["thermostats"]["nhc"]
    sysi = s["system_idx"].astype(np.int64)
    fn = _morse_fn(s["cell"], sysi)
    dt, kT = float(s["dt"]), float(s["kT"])
    np.testing.assert_allclose(oth.chain_masses(g["dof"], kT, g["tau"], 3), g["Q"][0],
                               rtol=1e-14)
    e0, f0 = fn(g["positions"][0])
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": f0, "energy": e0}
    ch = {"xi": g["xi"][0], "p_xi": g["p_xi"][0], "ke": g["KE"][0], "dof": g["dof"],
          "tau": g["tau"]}
    for k in range(1, g["positions"].shape[0]):
        st, ch = oth.nvt_nose_hoover_step(st, ch, fn, dt, kT, 3, 3, sysi)
        np.testing.assert_allclose(st["positions"], g["positions"][k], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(st["momenta"], g["momenta"][k], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(ch["xi"], g["xi"][k], rtol=1e-9, atol=1e-14)
        np.testing.assert_allclose(ch["p_xi"], g["p_xi"][k], rtol=1e-9, atol=1e-14)
        np.testing.assert_allclose(ch["ke"], g["KE"][k], rtol=1e-10)
        inv = oth.nose_hoover_invariant(st["energy"], s["masses"], st["momenta"], sysi,
                                        ch["xi"], ch["p_xi"], ch["q"], g["dof"], kT)
        np.testing.assert_allclose(inv, g["invariant"][k], rtol=1e-11)


def test_vrescale_oracle_matches_reference(golden):
    from oracle import thermostats as oth

    s, g = golden["thermostats"]["sys"], golden["thermostats"]["vr"]
    sysi = s["system_idx"].astype(np.int64)
    fn = _morse_fn(s["cell"], sysi)
    dt, kT = float(s["dt"]), float(s["kT"])
    e0, f0 = fn(g["positions"][0])
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": f0, "energy": e0}
    for k in range(1, g["positions"].shape[0]):
        st = oth.nvt_vrescale_step(st, fn, dt, kT, float(g["tau"]), g["r1"][k - 1],
                                   g["gamma"][k - 1], sysi)
        np.testing.assert_allclose(st["positions"], g["positions"][k], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(st["momenta"], g["momenta"][k], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(st["energy"], g["energy"][k], rtol=1e-10)


def _asym_force(r, zi, zj):
    return (1.0 + zi - 0.5 * zj) * (1.1 - r)


@pytest.mark.parametrize("case", ["plife", "asym"])
def test_pair_forces_oracle_matches_reference(golden, case):
    s, g = golden["pairforces"]["sys"], golden["pairforces"][case]
    if case == "plife":
        fn = lambda r, zi, zj: opair.particle_life_force(r, 1.0, 0.3, 1.0)  # noqa: E731
        cutoff = 1.2
    else:
        fn, cutoff = _asym_force, 1.1
    o = opair.pair_forces_forward(fn, s["positions"], np.transpose(s["cell"], (0, 2, 1)),
                                  np.array([True] * 3), s["system_idx"].astype(np.int64),
                                  s["atomic_numbers"].astype(np.float64), cutoff)
    for k in ("energy", "forces", "stress", "stresses"):
        np.testing.assert_allclose(o[k], g[k], rtol=1e-11, atol=1e-13)


def test_npt_langevin_isotropic_oracle_matches_reference(golden):
    from oracle import npt as onpt

    s, g = golden["npt"]["sys"], golden["npt"]["npt"]
    sysi = s["system_idx"].astype(np.int64)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q, cell_col):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(cell_col, (0, 2, 1)), np.array([True] * 3), sysi,
                               6.0)
        return o["energy"], o["forces"], o["stress"]

    dt, kT, p_ext = float(g["dt"]), float(g["kT"]), float(g["p_ext"])
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": g["forces"][0], "stress": g["stress"][0],
          "cell_positions": g["cell_positions"][0], "cell_velocities": g["cell_velocities"][0],
          "alpha": g["alpha"], "cell_alpha": g["cell_alpha"], "b_tau": g["b_tau"],
          "reference_cell": g["reference_cell"]}
    for k in range(1, g["positions"].shape[0]):
        st = onpt.npt_langevin_isotropic_step(st, fn, dt, kT, p_ext, g["cell_noise"][k - 1],
                                              g["particle_noise"][k - 1], sysi)
        for key, rt in (("positions", 1e-12), ("momenta", 1e-9), ("cell", 1e-12),
                        ("cell_positions", 1e-9), ("cell_velocities", 1e-9),
                        ("cell_masses", 1e-14), ("stress", 1e-9)):
            np.testing.assert_allclose(st[key], g[key][k], rtol=rt, atol=1e-14, err_msg=key)


@pytest.mark.parametrize("grp", ["crescale", "crescale_aniso", "crescale_tri",
                                 "crescale_tri_dev", "crescale_tri_avg"])
def test_npt_crescale_oracle_matches_reference(golden, grp):
    import functools

    from oracle import npt as onpt

    s, g = golden["crescale"]["sys"], golden["crescale"][grp]
    step = {"crescale": onpt.npt_crescale_isotropic_step,
            "crescale_aniso": onpt.npt_crescale_anisotropic_step,
            "crescale_tri": onpt.npt_crescale_triclinic_step,
            "crescale_tri_dev": onpt.npt_crescale_triclinic_step,
            "crescale_tri_avg": functools.partial(onpt.npt_crescale_triclinic_step,
                                                  average=True)}[grp]
    sysi = s["system_idx"].astype(np.int64)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q, cell_col):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(cell_col, (0, 2, 1)), np.array([True] * 3), sysi,
                               6.0)
        return o["energy"], o["forces"], o["stress"]

    dt, kT, tau = (float(g[k]) for k in ("dt", "kT", "tau"))
    p_ext = g["p_ext"]
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": g["forces"][0], "stress": g["stress"][0], "cell": g["cell"][0],
          "isothermal_compressibility": g["isothermal_compressibility"],
          "tau_p": g["tau_p"], "initial_cell_inv": np.linalg.inv(g["cell"][0]),
          "initial_volume": np.linalg.det(g["cell"][0])}
    for k in range(1, g["positions"].shape[0]):
        noise = (g["r1_a"][k - 1], g["gamma_a"][k - 1], g["cell_noise"][k - 1],
                 g["r1_b"][k - 1], g["gamma_b"][k - 1])
        st = step(st, fn, dt, kT, p_ext, tau, noise, sysi)
        for key in ("positions", "momenta", "cell", "stress", "energy"):
            # max|d| / max|ref| <= 1e-9: the triclinic steps amplify 1e-16 differences
            # of the matrix exponential to ~2e-10 over 8 steps
            np.testing.assert_allclose(st[key], g[key][k], rtol=0,
                                       atol=1e-9 * np.abs(g[key][k]).max(), err_msg=key)


def test_npt_langevin_anisotropic_oracle_matches_reference(golden):
    from oracle import npt as onpt

    s, g = golden["npt"]["sys"], golden["npt"]["npt_aniso"]
    sysi = s["system_idx"].astype(np.int64)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q, cell_col):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(cell_col, (0, 2, 1)), np.array([True] * 3), sysi,
                               6.0)
        return o["energy"], o["forces"], o["stress"]

    dt, kT = float(g["dt"]), float(g["kT"])
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": g["forces"][0], "stress": g["stress"][0], "cell": g["cell"][0],
          "cell_positions": g["cell_positions"][0], "cell_velocities": g["cell_velocities"][0],
          "alpha": g["alpha"], "cell_alpha": g["cell_alpha"], "b_tau": g["b_tau"],
          "reference_cell": g["reference_cell"]}
    for k in range(1, g["positions"].shape[0]):
        st = onpt.npt_langevin_anisotropic_step(st, fn, dt, kT, g["p_ext"], g["cell_noise"][k - 1],
                                                g["particle_noise"][k - 1], sysi)
        for key in ("positions", "momenta", "cell", "cell_positions", "cell_velocities",
                    "stress"):
            np.testing.assert_allclose(st[key], g[key][k], rtol=0,
                                       atol=1e-9 * np.abs(g[key][k]).max(), err_msg=key)


def test_npt_nose_hoover_isotropic_oracle_matches_reference(golden):
    from oracle import npt as onpt

    s, g = golden["npt"]["sys"], golden["npt"]["npt_nh"]
    sysi = s["system_idx"].astype(np.int64)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)

    def fn(q, cell_col):
        o = opair.pair_forward(opair.MORSE, tab, np.zeros(len(q), int), q,
                               np.transpose(cell_col, (0, 2, 1)), np.array([True] * 3), sysi,
                               6.0)
        return o["energy"], o["forces"], o["stress"]

    dt, kT, p_ext = float(g["dt"]), float(g["kT"]), float(g["p_ext"])
    st = {"positions": g["positions"][0], "momenta": g["momenta"][0], "masses": s["masses"],
          "forces": g["forces"][0], "stress": g["stress"][0], "reference_cell": g["cell"][0],
          "cell_position": g["cell_position"][0], "cell_momentum": g["cell_momentum"][0][:, 0],
          "t_xi": g["thermostat_positions"][0], "t_pxi": g["thermostat_momenta"][0],
          "t_ke": g["thermostat_kinetic_energy"][0], "t_tau": np.full(3, 10 * dt),
          "b_xi": g["barostat_positions"][0], "b_pxi": g["barostat_momenta"][0],
          "b_ke": g["barostat_kinetic_energy"][0], "b_tau": np.full(3, 100 * dt),
          "chain_steps": 2, "sy_steps": 3}
    for k in range(1, g["positions"].shape[0]):
        st = onpt.npt_nose_hoover_isotropic_step(st, fn, dt, kT, p_ext, sysi)
        for key, ref in (("positions", "positions"), ("momenta", "momenta"), ("cell", "cell"),
                         ("cell_position", "cell_position"), ("stress", "stress"),
                         ("t_xi", "thermostat_positions"), ("t_pxi", "thermostat_momenta"),
                         ("b_xi", "barostat_positions"), ("b_pxi", "barostat_momenta"),
                         ("t_q", "thermostat_masses"), ("b_q", "barostat_masses")):
            np.testing.assert_allclose(st[key], g[ref][k], rtol=0,
                                       atol=1e-9 * np.abs(g[ref][k]).max(), err_msg=key)
        np.testing.assert_allclose(st["cell_momentum"], g["cell_momentum"][k][:, 0], rtol=1e-9,
                                   atol=1e-12)
