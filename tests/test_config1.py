"""The oracle on the 256-atom Lennard-Jones argon NVE case, pinned to the
reference's own run (``tests/golden/config1.npz``, made by make_config1.py):
pair set, and the 100-step FP64 velocity-Verlet trajectory with both the
truncated and the energy-shifted LJ (torch_sim/integrators/nve.py:74-130,
lennard_jones.py:23-47, pair_potential.py:351-464)."""

import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import fused_md, neighbors as onl, pair as opair

SIGMA, EPS, RC = 3.405, 0.0104, 2.5 * 3.405


@pytest.fixture(scope="module")
def c1():
    return np.load(os.path.join(GOLDEN, "config1.npz"))


def test_oracle_pair_set_matches_reference(c1):
    cell_row = np.transpose(c1["init/cell"], (0, 2, 1))
    got = onl.neighbor_list(c1["init/positions"], cell_row, c1["init/pbc"], RC,
                            c1["init/system_idx"])
    ref = onl.sort_pairs(c1["pairs/ij"].astype(np.int64), np.zeros(c1["pairs/ij"].shape[1], int),
                         c1["pairs/shifts"].astype(np.float64))
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(np.rint(got[2]).astype(int), ref[2].astype(int))


@pytest.mark.parametrize("name", ["lj", "lj_shift"])
def test_oracle_nve_trajectory_matches_reference(c1, name):
    shift = float(c1["shift"]) if name == "lj_shift" else 0.0
    tab = opair.single_table(opair.LJ, SIGMA, EPS, eshift=shift)
    cell_row = np.transpose(c1["init/cell"], (0, 2, 1))
    sysi = c1["init/system_idx"]
    x, p, f = c1[f"{name}/positions"][0], c1[f"{name}/momenta"][0], c1[f"{name}/forces0"]
    every = int(c1["every"])
    for k in range(1, c1[f"{name}/positions"].shape[0]):
        o = fused_md.run(opair.LJ, tab, np.zeros(len(x), int), x, p, f, c1["init/masses"],
                         cell_row, sysi, RC, every, float(c1["dt"]), integrator="nve",
                         skin=1.0)
        x, p, f = o["positions"], o["momenta"], o["forces"]
        np.testing.assert_allclose(x, c1[f"{name}/positions"][k], rtol=0, atol=1e-9)
        np.testing.assert_allclose(p, c1[f"{name}/momenta"][k], rtol=1e-7, atol=1e-9)
        np.testing.assert_allclose(o["energy"][0], c1[f"{name}/epot"][k * every], rtol=1e-10)
        np.testing.assert_allclose(o["stress"][0], c1[f"{name}/stress"][k * every], rtol=1e-8,
                                   atol=1e-12)
    np.testing.assert_allclose(f, c1[f"{name}/forces_end"], rtol=1e-7, atol=1e-10)
