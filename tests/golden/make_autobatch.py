"""Generate ``autobatch.npz``: bins of the reference's ``to_constant_volume_bins``
(torch_sim/autobatching.py:46-144) for seeded random weights, and its memory
scalers (autobatching.py:305-420) for a seeded Cu batch.

    python tests/golden/make_autobatch.py /path/to/torch-sim
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)

from make_golden import _install_shims  # noqa: E402


def main(ref_root):
    _install_shims(ref_root)
    sys.path.insert(0, os.path.join(REPO, "torch-sim_b200"))
    import torch

    torch.set_default_dtype(torch.float64)
    import torch_sim as ts
    from torch_sim.autobatching import calculate_memory_scalers, to_constant_volume_bins

    from tsb import workloads as W

    rng = np.random.default_rng(77)
    out = {}
    for k in range(6):
        n = int(rng.integers(5, 60))
        w = rng.integers(1, 50, n).astype(float) if k % 2 else rng.uniform(0.1, 10.0, n)
        cap = float(w.max() * rng.uniform(1.0, 4.0))
        bins = to_constant_volume_bins(dict(enumerate(w.tolist())), cap)
        out[f"case{k}/weights"] = w
        out[f"case{k}/max_volume"] = np.array(cap)
        # bins as (bin id per item), in the reference's bin order
        bid = np.full(n, -1)
        for b, d in enumerate(bins):
            for key in d:
                bid[key] = b
        out[f"case{k}/bin_of_item"] = bid
        lst = to_constant_volume_bins(w.tolist(), cap)
        out[f"case{k}/list_bin_sums"] = np.array([sum(b) for b in lst])
    d = W.copper_batch(12, 8, 512, seed=3)
    T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt)  # noqa: E731
    st = ts.SimState(positions=T(d["positions"]), masses=T(d["masses"]), cell=T(d["cell"]),
                     pbc=T(d["pbc"], torch.bool),
                     atomic_numbers=T(d["atomic_numbers"], torch.long),
                     system_idx=T(d["system_idx"], torch.long))
    out["cu/scalers_density"] = np.array(calculate_memory_scalers(st, "n_atoms_x_density"))
    out["cu/scalers_atoms"] = np.array(calculate_memory_scalers(st, "n_atoms"))
    np.savez_compressed(os.path.join(HERE, "autobatch.npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
