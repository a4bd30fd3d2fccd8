"""mppnp's diffusive mixing step on the GPU (nuppn_mix_diffusion*) against the oracle's restatement
of mixdiff08: equal bit for bit (the device performs tridag's operations in its order), in both
matrix forms, with the limiter active, through host buffers in both layouts (rows of species, and
mppnp's yps(msl, nsp) columns of shells), and on device tensors in both layouts with strides above
the array's extent (a column slice of wider rows; the transpose of a [nsp, msl] array with msl > m).
The device calls run in a child process (its own CUDA context), which writes its results for this
process to compare."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys, importlib
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
solver = importlib.import_module("nuppn_modular2-ininet3_b200.solver")
case = np.load(sys.argv[2])
out = {}
for mesa in (0, 1):
    kw = dict(dq=case["dq"]) if mesa else dict(xm=case["xm"])
    for k, sig in enumerate((1e30, 50.0)):
        X, d = solver.mix_diffusion(case["X"], case["d"], 1.0e4, sig, consider=case["cons"], **kw)
        out[f"X_{mesa}_{k}"], out[f"d_{mesa}_{k}"] = X, d
big = np.full((case["X2"].shape[0], 304), 7.0)
big[:, :300] = case["X2"]
t = torch.tensor(big, dtype=torch.float64, device="cuda")
out["d_dev"] = solver.mix_diffusion_device(t[:, :300], case["d2"], 2.0e3, 1e30, xm=case["xm2"], consider=case["cons2"])
torch.cuda.synchronize()
out["X_dev"] = t.cpu().numpy()
Xf = np.asfortranarray(case["X"])
out["X_f"], out["d_f"] = solver.mix_diffusion(Xf, case["d"], 1.0e4, 50.0, consider=case["cons"], xm=case["xm"])
out["f_order"] = np.array(np.isfortran(out["X_f"]))
yps = np.full((300, 136), 5.0)  # [nsp][msl]: column s holds species s over msl >= m shells
yps[:, :128] = case["X2"].T
ty = torch.tensor(yps, dtype=torch.float64, device="cuda")
out["d_yps"] = solver.mix_diffusion_device(ty[:, :128].t(), case["d2"], 2.0e3, 1e30, dq=case["dq2"], consider=case["cons2"])
torch.cuda.synchronize()
out["yps"] = ty.cpu().numpy()
np.savez(sys.argv[3], **out)
'''


def _case(seed, m, nsp):
    rng = np.random.default_rng(seed)
    return (np.cumsum(rng.uniform(0.001, 0.01, m)), rng.uniform(1e-5, 1e-3, m), 10.0 ** rng.uniform(-6, 3, m),
            10.0 ** rng.uniform(-30, 0, (m, nsp)), rng.random(nsp) < 0.9)


def test_mixing_equals_oracle(orc, tmp_path):
    xm, dq, d, X, cons = _case(7, 400, 1109)
    xm2, dq2, d2, X2, cons2 = _case(8, 128, 300)
    np.savez(tmp_path / "case.npz", xm=xm, dq=dq, d=d, X=X, cons=cons, xm2=xm2, dq2=dq2, d2=d2, X2=X2, cons2=cons2)
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT, str(tmp_path / "case.npz"), str(tmp_path / "out.npz")],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.load(tmp_path / "out.npz")
    for mesa in (0, 1):
        kw = dict(dq=dq) if mesa else dict(xm=xm)
        for k, sig in enumerate((1e30, 50.0)):
            want, dw, st = orc.mix_diffusion(X, d, 1.0e4, sig, consider=cons, **kw)
            assert st == 0
            assert np.array_equal(got[f"X_{mesa}_{k}"], want) and np.array_equal(got[f"d_{mesa}_{k}"], dw)
    want, dw, st = orc.mix_diffusion(X2, d2, 2.0e3, 1e30, xm=xm2, consider=cons2)
    assert st == 0
    assert np.array_equal(got["X_dev"][:, :300], want) and np.array_equal(got["d_dev"], dw)
    assert (got["X_dev"][:, 300:] == 7.0).all()  # the row padding is not touched
    want, dw, st = orc.mix_diffusion(X, d, 1.0e4, 50.0, consider=cons, xm=xm)
    assert bool(got["f_order"]) and np.array_equal(got["X_f"], want) and np.array_equal(got["d_f"], dw)
    want, dw, st = orc.mix_diffusion(X2, d2, 2.0e3, 1e30, dq=dq2, consider=cons2)
    assert st == 0
    assert np.array_equal(got["yps"][:, :128].T, want) and np.array_equal(got["d_yps"], dw)
    assert (got["yps"][:, 128:] == 5.0).all()  # shells past m are not touched
