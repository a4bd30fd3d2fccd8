"""mppnp's diffusive mixing (frames/mppnp/source/mixing.F90) on the CPU: the oracle's restatement of
mixdiff08 against an independent dense assembly of the same implicit diffusion step (backward error at
the rounding level, values to the systems' conditioning), in both matrix
forms (matrixdiffus on mass coordinates, matrixdiffus_mesa on shell masses) and with the coefficient
limiter active; the library's host part (the Lagrangian coefficient, the argument checks that need
no GPU) against the oracle."""
import numpy as np
import pytest


def _case(seed, m=60, nsp=40):
    rng = np.random.default_rng(seed)
    xm = np.cumsum(rng.uniform(0.01, 0.05, m))
    dq = rng.uniform(1e-4, 1e-2, m)
    d = 10.0 ** rng.uniform(-8, 2, m)
    d[rng.random(m) < 0.2] = 0.0
    X = rng.uniform(0, 1, (m, nsp))
    return xm, dq, d, X


def _dense(X, d, h, sig, xm=None, dq=None, consider=None):
    """The implicit step (1 - h L) X_new = X of mixing.F90, assembled densely with the routines'
    limiter, solved by numpy for every mixed species (0 .. nsp-2)."""
    m = X.shape[0]
    D = np.array(d, float)
    A = np.zeros((m, m))
    if dq is None:
        xr = xm[1] - xm[0]
        al = min(D[1] * h / xr ** 2, sig)
        A[0, 0], A[0, 1] = 1 + al, -al
        for j in range(1, m - 1):
            xl, xr = xm[j] - xm[j - 1], xm[j + 1] - xm[j]
            al = h / (0.5 * (xm[j + 1] - xm[j - 1]))
            if sig < D[j + 1] * al / xr:
                D[j + 1] = sig / al * xr
            A[j, j - 1], A[j, j], A[j, j + 1] = -D[j] * al / xl, 1 + (D[j + 1] / xr + D[j] / xl) * al, -D[j + 1] * al / xr
        xl = xm[m - 1] - xm[m - 2]
        al = D[m - 1] * h / xl ** 2
        A[m - 1, m - 2], A[m - 1, m - 1] = -al, 1 + al
    else:
        dr = np.zeros(m)
        lim = lambda al, t, c: sig / (al * t) if al * t * c > sig else c
        dr[1] = lim(h / dq[0], 1 / dq[0], D[1])
        A[0, 0], A[0, 1] = 1 + h / dq[0] * dr[1] / dq[0], -h / dq[0] * dr[1] / dq[0]
        for j in range(1, m - 1):
            al = h / (0.5 * (dq[j] + dq[j - 1]))
            dr[j + 1] = lim(al, 1 / dq[j], D[j + 1])
            A[j, j - 1] = -dr[j] / dq[j - 1] * al
            A[j, j] = 1 + (dr[j + 1] / dq[j] + dr[j] / dq[j - 1]) * al
            A[j, j + 1] = -dr[j + 1] / dq[j] * al
        al = h / dq[m - 1] ** 2
        A[m - 1, m - 2], A[m - 1, m - 1] = -al * D[m - 1], 1 + al * D[m - 1]
    out = X.copy()
    cols = [s for s in range(X.shape[1] - 1) if consider is None or consider[s]]
    out[:, cols] = np.linalg.solve(A, X[:, cols])
    return out, D, A, cols


@pytest.mark.parametrize("mesa", [False, True], ids=["xm", "dq"])
@pytest.mark.parametrize("sig", [1e30, 5.0], ids=["free", "limited"])
def test_oracle_mixing_matches_dense_solve(orc, mesa, sig):
    xm, dq, d, X = _case(1)
    cons = np.random.default_rng(2).random(X.shape[1]) < 0.8
    h = 3.0e3
    got, dl, st = orc.mix_diffusion(X, d, h, sig, xm=None if mesa else xm, dq=dq if mesa else None, consider=cons)
    want, dw, A, cols = _dense(X, d, h, sig, xm=None if mesa else xm, dq=dq if mesa else None, consider=cons)
    assert st == 0
    # the systems are stiff (D h / dx^2 up to ~1e8): the Thomas algorithm and a pivoted solve agree to
    # cond x eps; the oracle's own backward error is at the rounding level
    res = np.abs(A @ got[:, cols] - X[:, cols]).max(axis=0) / (np.abs(A) @ np.abs(got[:, cols])).max(axis=0)
    assert res.max() < 1e-14, res.max()
    assert np.allclose(got, want, rtol=1e-6, atol=1e-14)
    assert np.array_equal(got[:, -1], X[:, -1])  # the last slot is not mixed
    assert np.array_equal(got[:, ~np.append(cons[:-1], True)][:, :-1], X[:, ~np.append(cons[:-1], True)][:, :-1])
    if not mesa:
        assert np.array_equal(dl, dw)  # matrixdiffus limits D in place
        if sig < 1e30:
            assert (dl < d).any()
    else:
        assert np.array_equal(dl, d)  # matrixdiffus_mesa limits a copy


def test_d_lagrangian_library_and_oracle(orc, solver_mod):
    rng = np.random.default_rng(4)
    m = 50
    d_eul = 10.0 ** rng.uniform(-2, 12, m)
    d_eul[::7] = 0.0
    rho = 10.0 ** rng.uniform(-8, 3, m)
    rad = np.sort(10.0 ** rng.uniform(-3, 2, m))
    lib = solver_mod.mix_d_lagrangian(d_eul, rho, rad)
    ref = orc.mix_d_lagrangian(d_eul, rho, rad)
    assert np.array_equal(lib, ref)
    lr = np.concatenate([[np.log(rad[0])], 0.5 * (np.log(rad[1:]) + np.log(rad[:-1]))])
    lp = np.concatenate([[np.log(rho[0])], 0.5 * (np.log(rho[1:]) + np.log(rho[:-1]))])
    want = np.where(d_eul > 0, d_eul * 3.0589703419947736e-11 ** 2 * np.exp(2 * (2 * lr + lp)), 0.0)
    assert np.allclose(lib, want, rtol=1e-13, atol=0)


def test_mixing_argument_errors_need_no_gpu(solver_mod):
    xm, dq, d, X = _case(5, m=8, nsp=4)
    bad = xm.copy()
    bad[3] = bad[2]  # a shell of zero width
    with pytest.raises(solver_mod.NuppnError):
        solver_mod.mix_diffusion(X, d, 1e3, 1e30, xm=bad)
    with pytest.raises(solver_mod.NuppnError):
        solver_mod.mix_diffusion(X[:1], d[:1], 1e3, 1e30, xm=xm[:1])  # one shell
    with pytest.raises(solver_mod.NuppnError):
        solver_mod.mix_diffusion(X, d, 1e3, 1e30, dq=np.zeros_like(dq))  # dq(1) = 0


def test_mixing_layouts_need_no_gpu(solver_mod):
    """Rows of species and mppnp's columns of shells are the two layouts; the strides come from the
    array, and any other layout is refused before the GPU is touched."""
    m, nsp = 8, 5
    X = np.zeros((m, nsp))
    assert solver_mod._mix_strides(X.shape, X.strides) == (nsp, 1)
    F = np.asfortranarray(X)
    assert solver_mod._mix_strides(F.shape, F.strides) == (1, m)
    wide = np.zeros((m, nsp + 3))[:, :nsp]
    assert solver_mod._mix_strides(wide.shape, wide.strides) == (nsp + 3, 1)
    L = solver_mod.load_library()
    xm, dq, d, _ = _case(6, m=m, nsp=nsp)
    buf = np.zeros(4 * m * nsp)
    for sh, sp in ((2, 2), (nsp - 1, 1), (1, m - 1), (0, 1), (1, 0)):
        dd = d.copy()
        st = L.nuppn_mix_diffusion(m, nsp, buf.ctypes.data, sh, sp, xm.ctypes.data, None, dd.ctypes.data, 1e3, 1e30,
                                   0, None)
        assert st != 0 and b"shell" in L.nuppn_last_error()
        assert np.array_equal(dd, d)  # refused before d_lagr is limited
