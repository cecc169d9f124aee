"""The reciprocal the rate passes use instead of IEEE division (rcp_nr in
pass_common.cuh: two Newton-Raphson steps from the hardware's approximate
FP64 reciprocal) against CUDA's correctly rounded 1.0 / x, over the operand
ranges the passes give it and far beyond:

* r^2 + 0.01 h^2 (1e-9 .. 1e-3 for the decks here),
* P_a + P_b = 2 rho0 c0^2 + gamma (p_a + p_b) (1e4 .. 1e9),
* 1/rho_a + 1/rho_b (1e-4 .. 1e-2),
plus random mantissas over 1e-30 .. 1e30 and both signs.

Bar: at most one unit in the last place from the correctly rounded result."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulps(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_rcp_within_one_ulp_of_division():
    torch = pytest.importorskip("torch")
    from uph_b200 import _lib

    rng = np.random.default_rng(3)
    parts = [
        10.0 ** rng.uniform(-9, -3, 200000),  # r^2 + 0.01 h^2
        10.0 ** rng.uniform(4, 9, 200000),  # P_a + P_b
        10.0 ** rng.uniform(-4, -2, 200000),  # 1/rho_a + 1/rho_b
        10.0 ** rng.uniform(-30, 30, 400000) * rng.choice([-1.0, 1.0], 400000),
        np.array([1.0, 2.0, 0.5, 3.0, 7.0, 1.0 + 2.0 ** -52, 2.0 - 2.0 ** -51, 1e-300, 1e300]),
    ]
    x = np.concatenate(parts)
    d_x = torch.from_numpy(x).cuda()
    d_y = torch.empty_like(d_x)
    want = (1.0 / d_x).cpu().numpy()  # CUDA's IEEE division, round to nearest
    st = _lib.lib().uph_rcp_selftest(C.c_void_p(d_x.data_ptr()), C.c_void_p(d_y.data_ptr()), x.size,
                                     C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, _lib.lib().uph_last_error()
    got = d_y.cpu().numpy()
    u = _ulps(got, want)
    assert np.all(np.isfinite(got))
    assert u.max() <= 1, f"max {u.max()} ulp at x = {x[u.argmax()]!r}"
    # nearly always the correctly rounded value itself
    assert np.mean(u == 0) > 0.9
