"""nuppn_integrate_device_noalloc: batched integration that allocates no device memory.

The entry point is for callers that cannot call cudaMalloc while they step (a program that hands
all of the GPU's memory to its own allocator at start-up, or keeps device allocation, which can
synchronize the whole GPU, out of its time-step loop). Its workspace lives in a fixed static device
array instead of buffers the library allocates. This test calls it through the C ABI twice in a row
on the same inputs and checks each result against nuppn_integrate_device, at the parity tests'
tolerance (1e-6 relative for X > 1e-12, 1e-15 absolute below).
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


def test_noalloc_matches_integrate_device(solver_mod, abi, wl):
    import torch

    net = wl.network(300)
    zb = wl.heshell_batch(6, net=net, seed=11)
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
    for call in range(2):
        X, ye, dtw, ierr, stats, bd = fresh()
        st = fn(dev.h, nz, p(X), nsp, *[p(t) for t in ins], p(ye), p(dtw), p(ierr), p(stats), p(bd),
                stream)
        assert st == 0, dev.L.nuppn_last_error()
        torch.cuda.synchronize()
        Xn = X.cpu().numpy()
        big = ref[0] > 1e-12
        rel = (np.abs(Xn - ref[0])[big] / ref[0][big]).max()
        ab = np.abs(Xn - ref[0])[~big].max(initial=0.0)
        assert rel <= 1e-6 and ab <= 1e-15, (call, rel, ab)
        assert np.abs(ye.cpu().numpy() - ref[1]).max() <= 1e-12
        assert (ierr.cpu().numpy() == ref[2]).all()
        assert (stats.cpu().numpy() == ref[3]).all()
        assert (bd.cpu().numpy() == ref[4]).all()
