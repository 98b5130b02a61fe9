"""Generate ``nl500k.json``: digests of the reference's own neighbour list on
the 500,000-atom argon system (config 2), too large to store as pairs.

Run in a container where the reference source tree is present::

    python tests/golden/make_nl500k.py /path/to/torch-sim

The system: argon fcc 50x50x50 conventional cells (a = 5.26 A, cubic periodic
cell of 263 A), positions jittered by N(0, 0.1 A) from ``tsb.workloads.argon_fcc``
(seed 0), float64.  For the cutoff 8.5 A and the Verlet-list radius 9.5 A the
reference's ``torch_nl_linked_cell`` (torch_sim/neighbors/torch_nl.py:156-215)
gives the full pair set; recorded are the pair count and the SHA-256 of the
sorted packed keys (``oracle.neighbors.pair_set_digest``).  The oracle's cell
list is run on the same input and must give the same digest (checked here).
"""

from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref_root):
    sys.path.insert(0, HERE)
    from make_golden import _install_shims

    _install_shims(ref_root)
    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    sys.path.insert(0, REPO)
    import torch
    from torch_sim.neighbors.torch_nl import torch_nl_linked_cell

    from oracle import neighbors as onl
    from tsb import workloads as W

    torch.set_num_threads(os.cpu_count() or 1)
    d = W.argon_fcc((50, 50, 50), jitter=0.1, seed=0)
    pos = torch.as_tensor(d["positions"], dtype=torch.float64)
    cell_row = torch.as_tensor(d["cell"][0], dtype=torch.float64).T.contiguous()
    out = {"system": "argon fcc 50x50x50, a = 5.26 A, N(0, 0.1 A) jitter (seed 0), float64",
           "n_atoms": int(pos.shape[0]), "cutoffs": {}}
    for rc in (8.5, 9.5):
        m, _, sh = torch_nl_linked_cell(pos, cell_row, torch.ones(3, dtype=torch.bool), rc,
                                        torch.zeros(pos.shape[0], dtype=torch.long))
        dig, n = onl.pair_set_digest(m.numpy(), sh.numpy())
        del m, sh
        om, _, osh = onl.neighbor_list_cells(d["positions"], d["cell"][0].T, rc)
        odig, on = onl.pair_set_digest(om, osh)
        assert (dig, n) == (odig, on), "oracle and reference pair sets differ"
        out["cutoffs"][str(rc)] = {"n_pairs": n, "sha256": dig}
        print(rc, n, dig, flush=True)
    with open(os.path.join(HERE, "nl500k.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TORCH_SIM_REF", ""))
