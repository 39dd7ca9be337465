"""Host arrays larger than 8 MB reach the device through pinned staging
buffers filled by several host threads (csrc/host_copy.cu).  Checked on the
2M-node network: the uploaded CSR, and a solve with host b/x against the
same solve with device vectors, bit for bit."""
import ctypes as C

import numpy as np
import pytest

from blood_network_b200 import amg
from blood_network_b200.network import make_config

pytestmark = pytest.mark.gpu


def test_staged_uploads_and_downloads():
    import torch
    net = make_config("vascular_2m", keep_segments=False)
    assert net.data.nbytes > 8 << 20 and net.rhs.nbytes > 8 << 20
    S = amg.AMGSolver(net.n, net.indptr, net.indices, net.data)
    ia, ja, val = S.level(0)["A"]
    # the input is symmetric: (A + A^T)/2 keeps its entries, order and values
    assert np.array_equal(ia, net.indptr) and np.array_equal(ja, net.indices)
    assert np.asarray(val).tobytes() == net.data.tobytes()
    # host b and x (x0 from an array view at an offset: pageable, not 16-byte aligned)
    buf = np.zeros(net.n + 1)
    x0 = buf[1:]
    x_host, it = S.solve(net.rhs, x0=x0, tol=1e-8)
    d_b = torch.from_numpy(net.rhs).cuda()
    d_x = torch.zeros(net.n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    it2 = S.solve_device(d_b.data_ptr(), d_x.data_ptr(), tol=1e-8)
    torch.cuda.synchronize()
    assert it == it2 and it > 0
    assert x_host.tobytes() == d_x.cpu().numpy().tobytes()
    S.close()
