"""nuppn_integrate_device_noalloc: batched integration that allocates no device memory.

The entry point is for callers that cannot call cudaMalloc while they step (a program that hands
all of the GPU's memory to its own allocator at start-up, or keeps device allocation, which can
synchronize the whole GPU, out of its time-step loop). Its workspace lives in a fixed static device
array instead of buffers the library allocates. These tests call it through the C ABI twice in a row
on the same inputs and check each result against nuppn_integrate_device, at the parity tests'
tolerance (1e-6 relative for X > 1e-12, 1e-15 absolute below):

* 6 zones of the 300-species network (each CTA of the call integrates one zone);
* 96 zones of the 1109-species network, whose workspace slab (about 2.7 MB) fits some two dozen
  times in the static array: the call runs that many CTAs and each reuses its slab for zone after
  zone. Free device memory must not change across the call.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    vp, i32 = C.c_void_p, C.c_int32
    L.nuppn_integrate_device_noalloc.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate_device_noalloc.restype = i32
    return L.nuppn_integrate_device_noalloc


def _compare_two_calls(solver_mod, abi, net, zb, check_memory=False):
    import torch

    dev = solver_mod.NetworkSolver(net, abi.default_knobs(integration_method=1), device=0)
    fn = _bind(dev.L)
    cu = lambda a, dt=torch.float64: torch.tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    nz, nsp = zb.X.shape
    ins = [cu(zb.t9_0), cu(zb.t9_1), cu(zb.rho_0), cu(zb.rho_1)]

    def fresh():
        return (cu(zb.X), cu(zb.ye), cu(zb.dtwant), torch.zeros(nz, dtype=torch.int32, device="cuda"),
                torch.zeros(nz * 8, dtype=torch.int32, device="cuda"), torch.zeros(nz, dtype=torch.int32, device="cuda"))

    X, ye, dtw, ierr, stats, bd = fresh()
    dev.integrate_device(X, *ins, ye, dtw, ierr, stats, bd)
    torch.cuda.synchronize()
    ref = (X.cpu().numpy(), ye.cpu().numpy(), ierr.cpu().numpy(), stats.cpu().numpy(), bd.cpu().numpy())
    assert (ref[2] == 0).all()

    p = lambda t: C.c_void_p(t.data_ptr())
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    bufs = [fresh() for _ in range(2)]  # every device buffer of both calls exists before the first
    torch.cuda.synchronize()
    free0 = None
    for call in range(2):
        X, ye, dtw, ierr, stats, bd = bufs[call]
        if call == 1 and check_memory:
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
        st = fn(dev.h, nz, p(X), nsp, *[p(t) for t in ins], p(ye), p(dtw), p(ierr), p(stats), p(bd),
                stream)
        assert st == 0, dev.L.nuppn_last_error()
        torch.cuda.synchronize()
        if free0 is not None:
            assert torch.cuda.mem_get_info()[0] == free0, "the no-allocation call changed free device memory"
        Xn = X.cpu().numpy()
        big = ref[0] > 1e-12
        rel = (np.abs(Xn - ref[0])[big] / ref[0][big]).max()
        ab = np.abs(Xn - ref[0])[~big].max(initial=0.0)
        assert rel <= 1e-6 and ab <= 1e-15, (call, rel, ab)
        assert np.abs(ye.cpu().numpy() - ref[1]).max() <= 1e-12
        assert (ierr.cpu().numpy() == ref[2]).all()
        assert (stats.cpu().numpy() == ref[3]).all()
        assert (bd.cpu().numpy() == ref[4]).all()
    return dev


def test_noalloc_matches_integrate_device(solver_mod, abi, wl):
    net = wl.network(300)
    _compare_two_calls(solver_mod, abi, net, wl.heshell_batch(6, net=net, seed=11))


def test_noalloc_reuses_slabs_without_allocating(solver_mod, abi, wl):
    net = wl.network(1107)
    zb = wl.heshell_batch(96, net=net, seed=13)
    _compare_two_calls(solver_mod, abi, net, zb, check_memory=True)
