"""The reference-named entry points on the host: CPU tensors are refused loudly
(there is no CPU path), and the preconditioner matrix -- set-up linear algebra, as
the reference's ``torch.inverse`` -- matches the oracle's operator."""
import numpy as np
import pytest
import torch

import oracle
from conftest import rel_l2
from deltamic_b200.cuda_class import MeshFTCUDA
from deltamic_b200.mesh import icosphere
from deltamic_b200.optimize import VectorAdam, compute_precondition_matrix
from deltamic_b200.render import compute_spatial_frequency_grid


def test_meshftcuda_refuses_cpu_tensors():
    v, f = icosphere(1, 0.3)
    xi = compute_spatial_frequency_grid((8, 8, 8), [1.0, 1.0, 1.0])
    otf = torch.ones(8, 8, 8)
    with pytest.raises(RuntimeError, match="CUDA"):
        MeshFTCUDA.apply(torch.tensor(v, dtype=torch.float32), torch.tensor(f),
                         torch.ones(len(f)), *xi, otf, 0.5)
    with pytest.raises(TypeError):
        MeshFTCUDA.apply(torch.tensor(v, dtype=torch.float16), torch.tensor(f),
                         torch.ones(len(f)), *xi, otf, 0.5)


def test_meshftcuda_off_grid_axes_refuse_cpu_tensors():
    """Axes that are not centred grids take the explicit-list path; on CPU tensors
    it refuses as loudly as the grid path (there is no CPU path)."""
    v, f = icosphere(1, 0.3)
    xi = list(compute_spatial_frequency_grid((8, 8, 8), [1.0, 1.0, 1.0]))
    xi[1] = xi[1] ** 2  # not (2k - (n-1)) pi / L
    with pytest.raises(RuntimeError, match="CUDA"):
        MeshFTCUDA.apply(torch.tensor(v, dtype=torch.float32), torch.tensor(f),
                         torch.ones(len(f)), *xi, torch.ones(8, 8, 8), 0.5)


def test_fourier3d_cpp_shims_refuse_cpu_tensors():
    from deltamic_b200.fourier3d_cpp import backward_fourier3d_cpp, forward_fourier3d_cpp
    v, f = icosphere(1, 0.3)
    V, F = torch.tensor(v, dtype=torch.float32), torch.tensor(f)
    C, X = torch.ones(len(f)), torch.zeros(4, 3)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        forward_fourier3d_cpp(V, F, C, X)
    g = torch.zeros(4, dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="must be a CUDA tensor"):
        backward_fourier3d_cpp(V, F, C, g, g, X)


def test_vector_adam_refuses_cpu_parameters():
    p = torch.nn.Parameter(torch.zeros(4, 3))
    p.grad = torch.ones(4, 3)
    with pytest.raises(RuntimeError, match="CUDA"):
        VectorAdam([p], lr=1e-2).step()


def test_compute_precondition_matrix_matches_oracle():
    v, f = icosphere(1, 0.3)
    V = torch.tensor(v, dtype=torch.float64)
    P = compute_precondition_matrix(V, torch.tensor(f), 5.0)
    assert P.dtype == torch.float64
    assert rel_l2(P.numpy(), oracle.fit.precondition_matrix(f, len(v), 5.0)) < 1e-12


def test_vector_adam_adopts_a_reference_layout_state():
    """A state saved by the reference VectorAdam (optimize.py:225-257: ``step`` a
    Python int, ``g2`` the per-vertex moment repeated over [nv, 3]) loads into this
    optimiser and is brought into its layout; a state of another shape raises."""
    from deltamic_b200.optimize import _adopt_state
    p = torch.nn.Parameter(torch.zeros(5, 3))
    opt = VectorAdam([p], lr=1e-2)
    g1 = torch.arange(15, dtype=torch.float32).reshape(5, 3)
    g2v = torch.arange(5, dtype=torch.float32) + 0.5
    ref_state = {"state": {0: {"step": 7, "g1": g1.clone(),
                               "g2": g2v[:, None].repeat_interleave(3, dim=1)}},
                 "param_groups": [dict(opt.param_groups[0], params=[0])]}
    opt.load_state_dict(ref_state)
    st = opt.state[p]
    _adopt_state(st, p, vector=True)
    assert st["step"].dtype == torch.int64 and st["step"].tolist() == [7]
    assert torch.equal(st["g1"], g1)
    assert st["g2"].shape == (5,) and torch.equal(st["g2"], g2v)
    _adopt_state(st, p, vector=True)  # already in this layout: unchanged
    assert torch.equal(st["g2"], g2v) and st["step"].tolist() == [7]
    bad = {"step": 1, "g1": g1.clone(), "g2": torch.zeros(4)}
    with pytest.raises(ValueError, match="g2"):
        _adopt_state(bad, p, vector=True)
    with pytest.raises(ValueError, match="keys"):
        _adopt_state({"step": 1}, p, vector=True)
