"""pandora_nonlinear_static: the nonlinear term for callers that cannot allocate
device memory (code running inside a memory pool or budget it does not own, which
may not call cudaMalloc).  They bring their own input and output buffers; the
library's scratch is fixed __device__ storage sized for grids of at most 64 points
per direction.

Checked through the C-ABI, on two calls in a row (the scratch keeps the previous
call's contents), against the oracle and against pandora_nonlinear, the entry
point that works on its own allocations, at 48^3, at the 64^3 maximum and on an
anisotropic grid.  This file sorts last so that a run stopping at its first
failure has run everything else."""
import ctypes

import numpy as np
import pytest

from helpers import rel_l2_fields

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(48, 48, 48), (64, 64, 64), (64, 48, 32)])
def test_static_nonlinear_matches_oracle_and_allocating_entry_point(gpu_lib, dims):
    import torch
    import oracle as O
    p = gpu_lib.workload_params("iso_decay", 48)
    p.nodes_x, p.nodes_y, p.nodes_z = dims
    with gpu_lib.Simulation(p) as s:
        s.init_fluid()
        ref = s.nonlinear()                       # allocating entry point
        shape = s.shape
        u = s.get_state()
    o = O.Oracle(p)
    o.set_state(u)
    nl_o = o.nonlinear()
    o.close()
    L = gpu_lib.load()
    dev_u = [torch.from_numpy(np.ascontiguousarray(c).view(np.float64)).cuda() for c in u]
    for call in range(2):
        dev_n = [torch.full(dev_u[0].shape, float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
        torch.cuda.synchronize()
        st = L.pandora_nonlinear_static(ctypes.byref(p), *[ctypes.c_void_p(t.data_ptr()) for t in dev_u],
                                        *[ctypes.c_void_p(t.data_ptr()) for t in dev_n], None)
        assert st == 0, L.pandora_strerror(st)
        got = [t.cpu().numpy().view(np.complex128).reshape(shape) for t in dev_n]
        assert rel_l2_fields(got, nl_o) < 1e-13, (call, dims)
        assert rel_l2_fields(got, ref) < 1e-13, (call, dims)


def test_static_nonlinear_rejects_large_grids(gpu_lib):
    L = gpu_lib.load()
    p = gpu_lib.workload_params("iso_decay", 96)
    null = ctypes.c_void_p(0)
    one = ctypes.c_void_p(256)   # never dereferenced: the size check comes first
    st = L.pandora_nonlinear_static(ctypes.byref(p), one, one, one, one, one, one, null)
    assert st == -6
