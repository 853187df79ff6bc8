"""Host threads: two threads, each with its own stream, drive the fused stage at the same time
(ctypes releases the GIL for the library calls, so the calls overlap).  The library's shared
state on that path is the per-device flags recording that a kernel's shared-memory attribute is
set, and the per-thread error string; each case must end bit for bit where it ends when run
alone.  The seven-species cases and configurations 1 and 5 are used by no other test, so the
threads make the first launches of those kernels in the process."""
from __future__ import annotations

import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _state(dc):
    Q, r = dc.primitives()
    return dc.conserved(), Q, r


@pytest.mark.parametrize("tile", [1, 5])
def test_two_threads_two_streams(f3d, cuda_ok, tile):
    import torch
    S = f3d.solver_module()
    cases = [f3d.random_curvilinear(n=12, ns=7, seed=70 + i) for i in range(2)]
    par = [S.DeviceCase(c, tile=tile) for c in cases]
    torch.cuda.synchronize()
    start = threading.Barrier(len(par))
    errors = []

    def run(dc):
        try:
            st = torch.cuda.Stream()
            with torch.cuda.stream(st):
                start.wait(timeout=60)
                for _ in range(3):
                    dc.step()
            st.synchronize()
        except Exception as e:  # reported on the main thread
            errors.append(e)

    threads = [threading.Thread(target=run, args=(dc,)) for dc in par]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    assert not any(t.is_alive() for t in threads)
    for c, dc in zip(cases, par):
        alone = S.DeviceCase(c, tile=tile)
        for _ in range(3):
            alone.step()
        for a, b in zip(_state(dc), _state(alone)):
            assert np.array_equal(a, b), (tile, c.name)
