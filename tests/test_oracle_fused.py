"""Pin the trajectory oracle of the fused kernel (CPU only).

* Philox4x32-10 against the generator's published known-answer vectors
  (Salmon et al., SC'11; the Random123 distribution's test vectors).
* The list-based force oracle (``oracle.fused_md.VerletForces``: pairs listed
  at cutoff + skin, rebuilt after moves beyond skin/2) gives, at every step of a
  trajectory, the forces, energies and stresses of ``oracle.pair.pair_forward``
  with a fresh neighbour list -- which tests/test_oracle_golden.py pins to the
  reference's own outputs.
* The trajectory replay reproduces the reference's BAOAB/NVE steps from
  ``oracle.md`` when its own normals are fed back.
"""

import numpy as np
import pytest

from oracle import fused_md, md as omd, pair as opair, philox

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", KAT)
def test_philox_known_answers(ctr, key, expect):
    got = philox.philox4x32_10(*ctr, *key)
    assert tuple(int(v) for v in got) == expect


def test_fused_normals_are_standard_normal():
    z = philox.fused_normals(1234, np.arange(200_000), 7)
    assert abs(z.mean()) < 5e-3
    assert abs(z.var() - 1.0) < 1e-2
    # distinct counters give independent draws
    z2 = philox.fused_normals(1234, np.arange(200_000), 8)
    assert abs(np.corrcoef(z[:, 0], z2[:, 0])[0, 1]) < 1e-2


def _cu(n_sys=3, seed=4):
    from tsb import workloads

    d = workloads.copper_batch(n_sys, 8, 120, seed=seed, jitter=0.05)
    cell_row = np.transpose(d["cell"], (0, 2, 1)).copy()
    return d, cell_row


def test_verlet_oracle_equals_fresh_lists_along_a_trajectory():
    d, cell_row = _cu()
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)
    sp = np.zeros(len(d["masses"]), dtype=int)
    pbc = np.ones((cell_row.shape[0], 3), bool)
    vf = fused_md.VerletForces(opair.MORSE, tab, sp, cell_row, d["system_idx"], 6.0, skin=0.4)
    rng = np.random.default_rng(0)
    x = d["positions"].copy()
    for _ in range(12):
        x = x + rng.normal(0.0, 0.06, x.shape)  # ~0.1 A per step: several rebuilds
        got = vf(x)
        ref = opair.pair_forward(opair.MORSE, tab, sp, x, cell_row, pbc, d["system_idx"], 6.0)
        np.testing.assert_allclose(got["forces"], ref["forces"], rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(got["energy"], ref["energy"], rtol=1e-12)
        np.testing.assert_allclose(got["stress"], ref["stress"], rtol=1e-11, atol=1e-15)
    assert 2 <= vf.n_builds < 12


@pytest.mark.parametrize("integrator", ["nve", "nvt_langevin"])
def test_trajectory_replay_matches_step_oracle(integrator):
    from tsb import workloads

    d, cell_row = _cu(2, seed=9)
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)
    sp = np.zeros(len(d["masses"]), dtype=int)
    pbc = np.ones((cell_row.shape[0], 3), bool)
    sysi = d["system_idx"]
    m = d["masses"]
    kT = 1000 * workloads.KB_EV
    p0 = omd.initialize_momenta(m, sysi, kT, np.random.default_rng(3).normal(size=(len(m), 3)))
    f0 = opair.pair_forward(opair.MORSE, tab, sp, d["positions"], cell_row, pbc, sysi,
                            6.0)["forces"]
    dt, gamma, seed = 0.002 * workloads.METAL_TIME, 10.0 / workloads.METAL_TIME, 77
    out = fused_md.run(opair.MORSE, tab, sp, d["positions"], p0, f0, m, cell_row, sysi, 6.0,
                       6, dt, integrator=integrator, kT=kT, gamma=gamma, seed=seed,
                       counter=5, skin=0.5)

    def fn(q):
        o = opair.pair_forward(opair.MORSE, tab, sp, q, cell_row, pbc, sysi, 6.0)
        return o["energy"], o["forces"]

    st = {"positions": d["positions"].copy(), "momenta": p0, "masses": m, "forces": f0,
          "energy": np.zeros(2)}
    for k in range(6):
        if integrator == "nve":
            st = omd.nve_step(st, fn, dt)
        else:
            z = philox.fused_normals(seed, np.arange(len(m)), 5 + k)
            st = omd.nvt_langevin_step(st, fn, dt, kT, gamma, z, sysi)
    np.testing.assert_allclose(out["positions"], st["positions"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(out["momenta"], st["momenta"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(out["energy"], st["energy"], rtol=1e-11)


@pytest.mark.parametrize("cells,rc", [((4, 4, 4), 5.0), ((5, 4, 6), 6.3), ((6, 6, 6), 8.5)])
def test_cell_list_oracle_equals_all_pairs_oracle(cells, rc):
    """The cell-list restatement (for systems too large for all pairs) gives the
    all-pairs oracle's pair set exactly on sheared, jittered cells with atoms
    outside the cell."""
    from oracle import neighbors as onl
    from tsb import workloads

    d = workloads.argon_fcc(cells, jitter=0.1, seed=3)
    rng = np.random.default_rng(1)
    F = np.eye(3) + rng.normal(0, 0.02, (3, 3))
    pos = d["positions"] @ F.T + rng.normal(0, 2.0, d["positions"].shape)
    C = d["cell"][0].T @ F.T
    a = onl.neighbor_list_cells(pos, C, rc)
    b = onl.neighbor_list(pos, C[None], np.ones(3, bool), rc, np.zeros(len(pos), np.int64))
    assert np.array_equal(a[0], b[0])
    assert np.array_equal(np.rint(a[2]), np.rint(b[2]))
