"""dustb_cell_index_static: the cell index for callers that cannot allocate device memory
when they call it (a host code whose device memory all comes from a pool it reserved at
start-up, or one that must not make synchronising cudaMalloc/cudaFree calls inside its time
step).  Its scratch is a fixed device array inside the library instead of a caller buffer.

Checked through the C ABI against dustb_cell_index (caller scratch) on the same particles,
bit for bit (integer outputs), on two calls in a row with the particles moved in between
(the shared array keeps the last call's contents), and the size limit.  This file is
collected last so that a run stopping at the first failure has run everything else."""
import ctypes as C

import numpy as np
import pytest

from athenak_b200.mesh import uniform_mesh
from athenak_b200.inputs import make_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def static_index(dev):
    n, ncell = dev.npart, dev.mesh.ncell_active
    order = torch.full((max(n, 1),), -1, dtype=torch.int32, device=dev.device)
    cstart = torch.full((ncell + 1,), -7, dtype=torch.int32, device=dev.device)
    rc = dev.lib.dustb_cell_index_static(dev.pctx, order.data_ptr(), cstart.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream)
    return rc, order[:n], cstart


def test_cell_index_static_matches_caller_scratch_version():
    from athenak_b200 import capi
    from athenak_b200.drag import DeviceDust
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.01, 0.1], [1.0, 0.5], 3, seed=13, vel_noise=0.05)
    dev = DeviceDust(st, {})
    for call in range(2):
        ref_order, ref_cstart = dev.cell_index()
        rc, order, cstart = static_index(dev)
        torch.cuda.synchronize()
        assert rc == 0, capi.load().dustb_last_error()
        np.testing.assert_array_equal(order.cpu().numpy(), ref_order.cpu().numpy())
        np.testing.assert_array_equal(cstart.cpu().numpy(), ref_cstart.cpu().numpy())
        # move the particles (many change cells) before the second call
        dev.register_copy()
        dev.push_imex(1.0, 0.0, 2e-3, 0.0)
        dev.route()
    assert dev.error_word() == 0


def test_cell_index_static_rejects_oversized_inputs():
    from athenak_b200 import capi
    from athenak_b200.drag import DeviceDust
    ms = uniform_mesh((16, 16, 16), (8, 8, 8), 2, (-0.05,) * 3, (0.05,) * 3)
    st = make_state(ms, [0.1], [1.0], 1, seed=2)
    dev = DeviceDust(st, {})
    big = capi.DustbCtx.from_buffer_copy(dev.ctx)
    big.part.npart = 1 << 26          # 256 MiB of keys: more than the fixed array holds
    big.part.stride = 1 << 26
    order = torch.empty(4, dtype=torch.int32, device=dev.device)
    cstart = torch.empty(ms.ncell_active + 1, dtype=torch.int32, device=dev.device)
    rc = dev.lib.dustb_cell_index_static(C.byref(big), order.data_ptr(), cstart.data_ptr(),
                                         torch.cuda.current_stream().cuda_stream)
    assert rc == -3                    # DUSTB_ESCRATCH, nothing launched
    assert b"scratch bytes" in capi.load().dustb_last_error()
