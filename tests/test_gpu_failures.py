"""Failure handling without a GPU fault.

Allocation failures are injected on the host: nemo_debug_fail_alloc(n) makes
the n-th device or page-locked allocation of the library report
cudaErrorMemoryAllocation without allocating.  The reference stops the
program when an ALLOCATE fails (original/nemolite2d.f90:308); here every
create call must instead return NEMO_ERR_ALLOC, set no handle and leave no
device memory behind, and the library must stay usable afterwards.  Each
create is driven through every one of its allocations in turn.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NEMO_ERR_ALLOC = 3


@pytest.fixture(scope="module")
def nb():
    import nemo_b200
    return nemo_b200


def free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def _drive(lib, create, destroy, limit=200):
    """create() -> (status, handle) under a countdown of 1, 2, ... until a
    create succeeds without the failure firing.  Returns the number of
    allocation sites exercised."""
    ok = create()
    assert ok[0] == 0, ok
    destroy(ok[1])                 # first use: lazy driver state is in place now
    base = free_bytes()
    sites = 0
    for n in range(1, limit):
        lib.nemo_debug_fail_alloc(n)
        st, h = create()
        left = lib.nemo_debug_fail_alloc(0)
        if left > 0:               # the n-th allocation was never reached
            assert st == 0 and h, (n, st)
            destroy(h)
            assert free_bytes() == base, "leak after a successful create"
            break
        sites += 1
        assert st == NEMO_ERR_ALLOC, "allocation %d: status %d" % (n, st)
        assert not h, "allocation %d: a handle was returned" % n
        assert free_bytes() == base, "allocation %d: device memory leaked" % n
    else:
        pytest.fail("create did not complete within %d allocations" % limit)
    return sites


def test_nemo_create_fails_cleanly_at_every_allocation(nb):
    lib = nb.load(False)
    p = nb.default_params(jpi=300, jpj=200, rdt=20.0, cbfr=0.00015, visc=0.1, nbump=4, seed=3,
                          bump_amp=20.0, bump_wmin=5e3, bump_wmax=40e3)

    def create():
        h = ctypes.c_void_p()
        st = lib.nemo_create(ctypes.byref(p), ctypes.byref(h))
        return st, h.value

    sites = _drive(lib, create, lambda h: lib.nemo_destroy(ctypes.c_void_p(h)))
    assert sites >= 3  # slab, pinned checksum buffer, bathymetry tables
    # the library is usable afterwards and computes the same run
    a = nb.Model(p)
    b = nb.Model(p)
    a.step_n(1, 20)
    b.step_n(1, 20)
    np.testing.assert_array_equal(a.field(nb.SSHN), b.field(nb.SSHN))


def test_lazy_allocations_fail_cleanly(nb):
    """Allocations made after creation (the record staging buffer, the
    autotuner's state backup) report NEMO_ERR_ALLOC and leave the context
    usable."""
    import torch
    m = nb.Model(jpi=120, jpj=90, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.3)
    m.step_n(1, 10)
    lib = m.lib
    host = torch.zeros(3 * 120 * 90, dtype=torch.float64, pin_memory=True).numpy()
    lib.nemo_debug_fail_alloc(1)
    st = lib.nemo_record(m.h, nb._dptr(host))
    assert lib.nemo_debug_fail_alloc(0) == 0 and st == NEMO_ERR_ALLOC
    sch, ms = nb.Schedule(), ctypes.c_double()
    lib.nemo_debug_fail_alloc(1)
    st = lib.nemo_autotune(m.h, 2, ctypes.byref(sch), ctypes.byref(ms))
    assert lib.nemo_debug_fail_alloc(0) == 0 and st == NEMO_ERR_ALLOC
    ref = nb.Model(jpi=120, jpj=90, rdt=20.0, cbfr=0.00015, visc=0.1, amp_tide=0.3)
    ref.step_n(1, 10)
    m.step_n(11, 10)
    ref.step_n(11, 10)
    m.record(host)
    m.record_wait()
    np.testing.assert_array_equal(host.reshape(3, 90, 120)[0], ref.field(nb.SSHN))
    np.testing.assert_array_equal(m.field(nb.UN), ref.field(nb.UN))


def test_nemo_ens_create_fails_cleanly_at_every_allocation(nb):
    lib = nb.load(False)
    members = nb.generate_members(9, 3, side_min=40, side_max=200, amp_scale=0.2)
    arr = (nb.Member * len(members))(*members)
    common = nb.default_params(dx=1000.0, dy=1000.0, rdt=20.0, cbfr=0.00015, visc=0.1)

    def create():
        h = ctypes.c_void_p()
        st = lib.nemo_ens_create(ctypes.byref(common), arr, len(members), ctypes.byref(h))
        return st, h.value

    sites = _drive(lib, create, lambda h: lib.nemo_ens_destroy(ctypes.c_void_p(h)))
    assert sites >= 8
    e = nb.Ensemble(members, common=common)
    e.step_n(1, 10)
    assert np.all(np.isfinite(e.checksums()))


@pytest.mark.parametrize("train", [0, 1])
def test_nemo_sur_create_fails_cleanly_at_every_allocation(nb, train):
    from nemo_b200 import surrogate as sm
    lib = nb.load(False)
    cfg = sm.SurConfig()
    lib.nemo_sur_default_config(ctypes.byref(cfg))
    cfg.nblocks, cfg.batch, cfg.height, cfg.width, cfg.train = 1, 2, 128, 128, train

    def create():
        h = ctypes.c_void_p()
        st = lib.nemo_sur_create(ctypes.byref(cfg), ctypes.byref(h))
        return st, h.value

    sites = _drive(lib, create, lambda h: lib.nemo_sur_destroy(ctypes.c_void_p(h)))
    assert sites >= 10


def test_convolution_wait_runs_out_and_the_surrogate_recovers(nb):
    """A forward convolution whose first input row never arrives: CTA 0 leaves
    that load out (a wait on a barrier nothing completes, not a broken
    kernel).  Its waits give up at the shortened limit, the kernel lets its
    other copies and MMAs finish, frees its tensor memory and returns, and
    nemo_sur_predict reports NEMO_ERR_TIMEOUT.  The next call on the same
    surrogate computes exactly what a surrogate that never timed out does."""
    import time
    import torch
    from nemo_b200 import surrogate as sm
    lib = nb.load(False)
    N, H, W = 2, 8, 128
    g = torch.Generator(device="cuda").manual_seed(3)
    snap = torch.randn((N, H, W, 4), device="cuda", generator=g)
    tide = torch.randn((N,), device="cuda", generator=g)
    norm = ([1.0, 2.0, 0.5, 1.5], [0.0, 0.1, 0.0, 0.2], [1.0, 0.8, 1.2])
    sur = [sm.Surrogate(nblocks=1, batch=N, height=H, width=W, train=False, seed=4) for _ in range(2)]
    for s in sur:
        s.set_norm(*norm)
    outs = [torch.zeros(s.out_shape(N), device="cuda") for s in sur]
    torch.cuda.synchronize()
    assert lib.nemo_debug_conv_wait(1_000_000, 1) == 0  # 1 ms; the next forward launch omits a load
    try:
        t0 = time.perf_counter()
        with pytest.raises(nb.NemoError) as ei:
            sur[0].predict(snap.data_ptr(), tide.data_ptr(), N, outs[0].data_ptr())
        elapsed = time.perf_counter() - t0
    finally:
        lib.nemo_debug_conv_wait(0, 0)
    assert ei.value.status == 5, ei.value  # NEMO_ERR_TIMEOUT
    assert elapsed < 1.5, "the shortened limit was not used (%.2f s)" % elapsed
    for s, o in zip(sur, outs):
        s.predict(snap.data_ptr(), tide.data_ptr(), N, o.data_ptr())
    torch.cuda.synchronize()
    a, b = (o.cpu().numpy() for o in outs)
    assert np.all(np.isfinite(a)) and np.any(a)
    np.testing.assert_array_equal(a.view(np.int32), b.view(np.int32))

