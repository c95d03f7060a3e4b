"""The libtorch extension loads, registers torch.ops.sagittasbr.rcs with its schema,
and reports a missing GPU as a clean error (no compute without a GPU)."""
import numpy as np
import pytest
import torch

from sagittasbr_b200 import meshes as M


def test_extension_registers_the_operator():
    from sagittasbr_b200 import torch_ext
    ops = torch_ext.load()
    schema = str(ops.rcs.default._schema)
    assert schema.startswith("sagittasbr::rcs(Tensor verts, Tensor freqs, Tensor tris, Tensor theta, Tensor phi")
    assert schema.endswith("-> Tensor")


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU error path")
def test_without_gpu_the_operator_raises():
    from sagittasbr_b200 import torch_ext
    v, t = M.icosphere(1, 1.0)
    verts = torch.tensor(v, dtype=torch.float64, requires_grad=True)
    freqs = torch.tensor([1e9], dtype=torch.float64)
    with pytest.raises(RuntimeError, match="sbr_scene_create"):
        torch_ext.rcs(verts, t, [90.0], [0.0], freqs, 8, 8, 2.0, 2)


def test_operator_rejects_bad_shapes():
    from sagittasbr_b200 import torch_ext
    verts = torch.zeros(4, 2, dtype=torch.float64)
    with pytest.raises(RuntimeError, match="verts must be"):
        torch_ext.rcs(verts, np.zeros((1, 3)), [90.0], [0.0], torch.tensor([1e9]), 8, 8, 2.0, 2)
