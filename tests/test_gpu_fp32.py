"""FP32 factor with FP64 refinement (sm100_factor_dtype=torch.float32).

The factor and the substitutions run in FP32 and every solve is refined
against the FP64 operator.  Where the FP32 LDL^T stays positive definite the
polished fixed point and its gradients agree with the all-FP64 run (heads
within 1e-9 m, gradients within 1e-6 relative).  On networks whose node
matrix is too ill-conditioned for an FP32 factor (the 782-junction workload:
conductances spanning about 2e5 once the PRVs open, condition number about
1e11) a pivot loses positivity and the solve refuses with the FP32 factor
named, instead of returning a wrong answer."""
import numpy as np
import pytest
import torch

from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu

POLISHED_HEAD_ATOL_FT = 1e-9 / 0.3048


def _solve(net, cuda, dtype, d, rh, sens):
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    s.sm100_factor_dtype = dtype
    D = torch.tensor(d, device=cuda, requires_grad=True)
    R = s.r_hw.clone().requires_grad_(True)
    h, q, e = implicit_solve(s, D, torch.tensor(rh, device=cuda), r_hw=R, accuracy=1e-6)
    (h[:, sens] ** 2).sum().backward()
    return s, h.detach(), q.detach(), D.grad, R.grad


@pytest.mark.parametrize("which", ["config1", "small_looped"])
def test_fp32_factor_matches_fp64(cuda, which):
    net = synth.config1_network() if which == "config1" else synth.config3_networks()[0]
    B = 32
    d, _ = synth.config2_scenarios(net, B, seed=31, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    sens = synth.sensor_nodes(net, 8)
    _, h64, q64, gd64, gr64 = _solve(net, cuda, torch.float64, d, rh, sens)
    _, h32, q32, gd32, gr32 = _solve(net, cuda, torch.float32, d, rh, sens)
    assert float((h32 - h64).abs().max()) <= POLISHED_HEAD_ATOL_FT
    assert float((q32 - q64).abs().max()) <= 1e-9
    for a, b in ((gd32, gd64), (gr32, gr64)):
        assert float((a - b).abs().max()) <= 1e-6 * float(b.abs().max())


def test_fp32_factor_refuses_an_ill_conditioned_network(cuda):
    net = synth.config2_network()
    B = 8
    d, rh = synth.config2_scenarios(net, B, seed=31, sigma=0.3)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    s.sm100_factor_dtype = torch.float32
    with pytest.raises(RuntimeError, match="FP32"):
        implicit_solve(s, torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda),
                       accuracy=1e-6)
