"""The ``torch.ops.tsb`` operators without a GPU: registration, schemas, fake
kernels (shapes under FakeTensorMode, the neighbour list's data-dependent pair
count) and the loud failure on CPU tensors (no CPU kernel is registered)."""

import pytest
import torch


def _ops():
    from tsb import ops

    return ops


def test_every_operator_is_registered_with_its_mutations():
    ops = _ops()
    for name in ops.OPS:
        op = getattr(torch.ops.tsb, name)
        schema = op.default._schema
        mutated = [a.name for a in schema.arguments if a.alias_info and a.alias_info.is_write]
        # in-place operators (trailing underscore) declare what they write; the
        # functional ones write nothing
        assert bool(mutated) == name.endswith("_"), (name, mutated)


def test_fake_kernels_give_output_metadata():
    _ops()
    from torch._subclasses.fake_tensor import FakeTensorMode
    from torch.fx.experimental.symbolic_shapes import ShapeEnv

    with FakeTensorMode(shape_env=ShapeEnv()):
        f64 = dict(dtype=torch.float64, device="cuda")
        pos = torch.empty((10, 3), **f64)
        cell = torch.empty((2, 3, 3), **f64)
        pbc = torch.empty((2, 3), dtype=torch.uint8, device="cuda")
        sysi = torch.empty(10, dtype=torch.int64, device="cuda")
        tab = torch.empty((1, 1, 5), **f64)
        from tsb import _lib as L

        flags = L.OUT_FORCES | L.OUT_STRESS
        e, f, s, ea, sa = torch.ops.tsb.pair_forward(pos, cell, pbc, sysi, None, tab,
                                                     L.POT_MORSE, 1, 6.0, flags, 2, 5)
        assert (tuple(e.shape), tuple(f.shape), tuple(s.shape)) == ((2,), (10, 3), (2, 3, 3))
        assert ea.numel() == 0 and sa.numel() == 0 and e.device.type == "cuda"
        m, sm, sh = torch.ops.tsb.nl_build(pos, cell, pbc, sysi, 6.0, 0, 2, 0)
        assert m.shape[0] == 2 and m.dtype == torch.int64 and sh.dtype == torch.float64
        # the pair count is data-dependent: one unbacked symbol shared by the outputs
        assert str(m.shape[1]) == str(sm.shape[0]) == str(sh.shape[0])
        assert not isinstance(m.shape[1], int)
        torch.ops.tsb.md_kick_(pos, pos, sysi, torch.empty(2, **f64), 0.5)


def test_operators_refuse_cpu_tensors():
    _ops()
    p = torch.zeros((2, 3), dtype=torch.float64)
    with pytest.raises(NotImplementedError, match="CPU"):
        torch.ops.tsb.md_kick_(p, p, torch.zeros(2, dtype=torch.int64),
                               torch.zeros(1, dtype=torch.float64), 0.5)
