"""Real-to-complex and complex-to-real transforms (shafft_sm100_rplan_*)
against the CPU oracle: the R2C spectrum is the first L/2 + 1 frequencies of
the oracle's full DFT of the real input; C2R of a Hermitian half spectrum is
the unnormalised inverse DFT of the full spectrum (real).  Tolerances
(relative L2): 1e-6*log2(N) for float, 1e-14*log2(N) for double."""
import math

import numpy as np
import pytest

from oracle import oracle as o
from shafft_b200 import _sm100

pytestmark = pytest.mark.gpu

SHAPES = [(2,), (64,), (1000,), (6000,), (4096,), (16, 32, 64), (31, 48), (7, 5, 12), (3, 1, 8),
          (64, 64, 32), (17, 4098), (1, 30)]


def tol(n, prec):
    return (1e-14 if prec else 1e-6) * max(1.0, math.log2(max(n, 2)))


def _torch():
    return pytest.importorskip("torch")


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("dims", SHAPES)
def test_r2c_and_c2r_vs_oracle(dims, prec):
    torch = _torch()
    n = math.prod(dims)
    H = dims[-1] // 2
    rdt = np.float64 if prec else np.float32
    rng = np.random.Generator(np.random.MT19937(n))
    x = rng.uniform(-1, 1, size=dims).astype(rdt)
    plan = _sm100.RPlan(dims, prec)
    spec_n = plan.spectrum_elements
    assert spec_n == n // dims[-1] * (H + 1)
    cdt = torch.complex128 if prec else torch.complex64
    # R2C (the input buffer is scratch: keep a copy of x on the host)
    xin = torch.from_numpy(x.copy()).cuda()
    spec = torch.empty(spec_n, dtype=cdt, device="cuda")
    plan.r2c(xin.data_ptr(), spec.data_ptr(), 1.0, 0)
    torch.cuda.synchronize()
    full = o.fftn(x.astype(np.complex128), precise=bool(prec))
    ref = full[..., :H + 1]
    err = o.rel_l2(spec.cpu().numpy().reshape(ref.shape), ref)
    assert err <= tol(n, prec), ("r2c", dims, err)
    # C2R of the oracle's half spectrum: the unnormalised inverse is n * x
    sin = torch.from_numpy(np.ascontiguousarray(ref).astype(np.complex128 if prec else np.complex64)).cuda()
    y = torch.empty(n, dtype=torch.float64 if prec else torch.float32, device="cuda")
    plan.c2r(sin.data_ptr(), y.data_ptr(), 1.0 / n, 0)
    torch.cuda.synchronize()
    err = o.rel_l2(y.cpu().numpy().reshape(dims), x)
    assert err <= tol(n, prec), ("c2r", dims, err)
    # round trip through the library alone, scale fused into the C2R
    xin = torch.from_numpy(x.copy()).cuda()
    plan.r2c(xin.data_ptr(), spec.data_ptr(), 1.0, 0)
    plan.c2r(spec.data_ptr(), y.data_ptr(), 1.0 / n, 0)
    torch.cuda.synchronize()
    assert o.rel_l2(y.cpu().numpy().reshape(dims), x) <= tol(n, prec)
    plan.destroy()


def test_r2c_headline_sized_cube():
    """256^3 float: R2C then C2R with the normalisation fused returns the
    input; the spectrum's DC term is the sum of the input."""
    torch = _torch()
    dims = (256, 256, 256)
    n = math.prod(dims)
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.rand(n, device="cuda", generator=g) * 2 - 1
    x0 = x.clone()
    plan = _sm100.RPlan(dims, 0)
    spec = torch.empty(plan.spectrum_elements, dtype=torch.complex64, device="cuda")
    plan.r2c(x.data_ptr(), spec.data_ptr(), 1.0, 0)
    y = torch.empty_like(x)
    dc = complex(spec[0].item())
    plan.c2r(spec.data_ptr(), y.data_ptr(), 1.0 / n, 0)
    torch.cuda.synchronize()
    err = float((torch.linalg.vector_norm(y - x0) / torch.linalg.vector_norm(x0)).item())
    assert err <= tol(n, 0), err
    total = float(x0.double().sum().item())
    assert abs(dc.real - total) <= 1e-4 * math.sqrt(n) and abs(dc.imag) <= 1e-4 * math.sqrt(n)
    plan.destroy()
