"""adm_vmult_host with pinned host buffers runs the z-slab pipeline (copies
overlapped with the tiles of each slab, atomic node sums); with pageable
buffers it runs the plain path. Both must match the device vmult and the
oracle."""
import numpy as np
import pytest
import torch

from pairs import CASES, make_case, make_gpu, make_oracle, rel_max

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_pinned_pipeline_matches_device_vmult(name):
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g1, g2 = make_gpu(cfg, cells), make_gpu(cfg, cells)
    for g in (g1, g2):
        g.set_time(3e-5)
    o.set_time(3e-5)
    src = g1.from_grid(T)
    dst = g1.initialize_dof_vector()
    src_h = torch.empty(g2.m(), dtype=torch.float64).pin_memory()
    dst_h = torch.empty(g2.m(), dtype=torch.float64).pin_memory()
    src_h.copy_(src.cpu())
    for _ in range(2):  # the phase history advances in both handles alike
        g1.vmult(dst, src)
        g2.vmult_host(src_h.numpy(), dst_h.numpy())
        ref = o.vmult(np.asarray(T).reshape(-1))
        got = dst_h.numpy()
        assert rel_max(got, dst.cpu().numpy()) <= 1e-13
        assert rel_max(g2.to_grid(torch.from_numpy(got.copy())).reshape(-1), ref) <= 1e-12
    # pageable buffers: the plain path
    plain = g2.vmult_host(src_h.numpy().copy())
    g1.vmult(dst, src)
    assert rel_max(plain, dst.cpu().numpy()) <= 1e-13
    assert g2.device_error() == 0
