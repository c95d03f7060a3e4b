"""The libtorch extension of the sweep: `torch.ops.sagittasbr.rcs`, a C++
torch::autograd::Function (csrc/torch_rcs.cpp) over libsbr's C ABI.

sigma [n_angles, n_freqs] (m^2) is differentiable with respect to the vertices
([V, 3]) and the frequencies ([n_freqs], Hz); backward runs sbr_adjoint along the
frozen hit paths.  Built by `make -C sagittasbr_b200/csrc torch` into
sagittasbr_b200/libsbr_torch.so; there is no fallback when it is missing.
"""
from __future__ import annotations

import os

import torch

from . import PREC_MIXED, lib

HERE = os.path.dirname(os.path.abspath(__file__))
EXT_PATH = os.path.join(HERE, "libsbr_torch.so")
_loaded = False


def load():
    """Loads the extension (and libsbr first) and returns the `torch.ops.sagittasbr` namespace."""
    global _loaded
    if not _loaded:
        if not os.path.exists(EXT_PATH):
            raise RuntimeError(f"{EXT_PATH} is not built; run `make -C sagittasbr_b200/csrc torch`")
        lib()
        torch.ops.load_library(EXT_PATH)
        _loaded = True
    return torch.ops.sagittasbr


def rcs(verts: torch.Tensor, tris, theta, phi, freqs: torch.Tensor, nx: int, ny: int, grid: float,
        max_bounces: int, reflection_const: float = 1.0, precision: int = PREC_MIXED) -> torch.Tensor:
    """Differentiable sigma [n_angles, n_freqs] of the mesh through the C++ autograd Function."""
    ops = load()
    t = torch.as_tensor(tris, dtype=torch.int64)
    th = torch.as_tensor(theta, dtype=torch.float64)
    ph = torch.as_tensor(phi, dtype=torch.float64)
    return ops.rcs(verts, freqs, t, th, ph, int(nx), int(ny), float(grid), int(max_bounces), float(reflection_const),
                   int(precision))
