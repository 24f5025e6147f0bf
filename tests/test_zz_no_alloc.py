"""The allocation-free checksum entry point against the allocating one.

nemo_checksums_noalloc serves callers that cannot call cudaMalloc: hosts whose
device memory is all owned by their own pool, or loops that must not pay a
cudaMalloc's implicit synchronisation.  It takes plain device pointers and
keeps its scratch in a fixed array inside the library.  This file is collected
last so that a failure here leaves every other test already run; it passes
alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_checksums_match_allocating_entry_point_twice():
    import torch
    import nemo_b200 as nb

    lib = nb.load(False)
    kw = dict(jpi=333, jpj=517, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.2, nbump=6,
              seed=11, bump_amp=20.0, bump_wmin=5e3, bump_wmax=60e3, device=0)
    m = nb.Model(strict=False, **kw)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")  # caller-owned output
    for call, (istp0, n) in enumerate([(1, 40), (41, 25)]):
        m.step_n(istp0, n)
        m.sync()
        ref = m.checksums()                                  # allocating path
        ptrs = []
        for fid in (nb.SSHN, nb.UN, nb.VN):
            base, pitch = m.device_field(fid)
            # element (1,1): (jj+1)*pitch + (ji+2) doubles from the base
            ptrs.append(base + 8 * (2 * pitch + 3))
        arr = (ctypes.c_void_p * 3)(*ptrs)
        st = lib.nemo_checksums_noalloc(arr, 3, m.jpi, m.jpj, pitch, out.data_ptr(), None)
        assert st == 0, "call %d status %d" % (call, st)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # same fixed reduction order as nemo_checksums: the same bits
        np.testing.assert_array_equal(got.view(np.int64), ref.view(np.int64),
                                      err_msg="call %d" % call)
        assert np.all(got > 0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    import nemo_b200 as nb

    lib = nb.load(False)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    arr = (ctypes.c_void_p * 1)(buf.data_ptr())
    assert lib.nemo_checksums_noalloc(arr, 1, 4, 16385, 4, out.data_ptr(), None) == 1
    assert lib.nemo_checksums_noalloc(arr, 5, 4, 2, 4, out.data_ptr(), None) == 1
