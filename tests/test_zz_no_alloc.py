"""lsb_solve_noalloc through the C ABI: the solve for callers that cannot call cudaMalloc
(code running under a framework that owns all device memory, or that must avoid
cudaMalloc's implicit synchronisation). Its scratch lives in a static device array of
the library; the result must equal lsb_solve's (FP32 precision, same stop rule) within
the parity tolerance used by the other GPU tests, on two calls in a row, and the second
call must not change the device's free memory (nothing is allocated).

Collected last on purpose (file name), so a failure here does not hide the others; it
also passes when run alone in a fresh process.
"""

import ctypes

import numpy as np
import pytest

from tests.conftest import reference_material

pytestmark = pytest.mark.gpu

EXT = (1.2, 0.8, 0.9)
EPS_BAR = np.array([[2.1, 0.9, 0.8, 0.4, 0.9, 0.5],
                    [1.0, 0.0, 0.0, 0.0, 0.0, 0.0]], dtype=np.float32)


def relmax(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / np.abs(b).max()


def call_noalloc(lib, _lib, n, lm_d, mu_d, eb, eps, sig, stream):
    b = eb.shape[0]
    vox = np.array(n, dtype=np.int32)
    ext = np.array(EXT, dtype=np.float64)
    iters = np.zeros(b, np.int32)
    status = np.zeros(b, np.int32)
    resid = np.zeros(b, np.float64)
    mean = np.zeros((b, 6), np.float64)
    rc = lib.lsb_solve_noalloc(
        vox.ctypes.data_as(_lib.c_int_p), ext.ctypes.data_as(_lib.c_double_p), b,
        ctypes.c_void_p(lm_d.data_ptr()), ctypes.c_void_p(mu_d.data_ptr()),
        eb.ctypes.data_as(_lib.c_float_p), ctypes.c_void_p(eps.data_ptr()),
        ctypes.c_void_p(sig.data_ptr()), mean.ctypes.data_as(_lib.c_double_p), 1e-20, 1e-5,
        60, iters.ctypes.data_as(_lib.c_int_p), status.ctypes.data_as(_lib.c_int_p),
        resid.ctypes.data_as(_lib.c_double_p), ctypes.c_void_p(stream))
    _lib.check(rc, "lsb_solve_noalloc")
    return iters, status, mean


@pytest.mark.parametrize("n,side_stream", [((32, 32, 16), False), ((24, 20, 18), True)])
def test_noalloc_matches_lsb_solve(built_library, n, side_stream):
    import torch

    from jaxmaterials_b200 import GridSpec, _lib
    from jaxmaterials_b200.solver import RULE_CUDA, Solver

    lib = _lib.load()
    g = GridSpec(*n, *EXT)
    lm, mu = reference_material(n)
    lm_d = torch.as_tensor(lm, dtype=torch.float32, device="cuda")
    mu_d = torch.as_tensor(mu, dtype=torch.float32, device="cuda")
    b = EPS_BAR.shape[0]

    ref_solver = Solver(g, batch=b, precision="fp32")
    ref = ref_solver.solve(lm_d, mu_d, EPS_BAR, rtol=1e-20, atol=1e-5, maxiter=60, rule=RULE_CUDA)
    torch.cuda.synchronize()

    eb = np.ascontiguousarray(EPS_BAR)
    # outputs allocated once, before the calls: the calls themselves must allocate nothing
    eps = torch.empty((b, 6) + n, dtype=torch.float32, device="cuda")
    sig = torch.empty_like(eps)
    stream = torch.cuda.Stream() if side_stream else None
    handle = stream.cuda_stream if stream is not None else 0
    results = []
    free_after = []
    for _ in range(2):
        eps.fill_(float("nan"))
        sig.fill_(float("nan"))
        torch.cuda.synchronize()
        iters, status, mean = call_noalloc(lib, _lib, n, lm_d, mu_d, eb, eps, sig, handle)
        torch.cuda.synchronize()
        free_after.append(torch.cuda.mem_get_info()[0])
        assert np.array_equal(iters, ref.iters)
        assert np.array_equal(status, ref.status)
        assert relmax(eps.cpu().numpy(), ref.epsilon.cpu().numpy()) < 2e-5
        assert relmax(sig.cpu().numpy(), ref.sigma.cpu().numpy()) < 2e-5
        assert relmax(mean, ref.mean_sigma) < 1e-5
        results.append(eps.cpu().numpy())
    assert relmax(results[1], results[0]) < 2e-5
    # the second call (scratch address and tables already set up) allocated no device memory
    assert free_after[1] == free_after[0]
    ref_solver.close()


def test_noalloc_rejects_oversized_problem(built_library):
    import torch

    from jaxmaterials_b200 import _lib

    lib = _lib.load()
    vox = np.array([128, 128, 128], dtype=np.int32)
    ext = np.array([1.0, 1.0, 1.0], dtype=np.float64)
    eb = np.zeros(36, np.float32)
    iters = np.zeros(6, np.int32)
    status = np.zeros(6, np.int32)
    # small valid device buffers: the size check rejects the call before any launch, and
    # even a launch would only touch memory that exists
    buf = torch.zeros(16, dtype=torch.float32, device="cuda")
    ptr = ctypes.c_void_p(buf.data_ptr())
    rc = lib.lsb_solve_noalloc(vox.ctypes.data_as(_lib.c_int_p), ext.ctypes.data_as(_lib.c_double_p),
                               6, ptr, ptr, eb.ctypes.data_as(_lib.c_float_p), ptr, None,
                               None, 1e-6, 0.0, 10, iters.ctypes.data_as(_lib.c_int_p),
                               status.ctypes.data_as(_lib.c_int_p), None, None)
    assert rc < 0
    assert b"scratch" in lib.lsb_last_error()
    # batch above LSB_NOALLOC_MAX_BATCH
    vox = np.array([4, 4, 4], dtype=np.int32)
    eb = np.zeros(6 * 65, np.float32)
    it = np.zeros(65, np.int32)
    stt = np.zeros(65, np.int32)
    rc = lib.lsb_solve_noalloc(vox.ctypes.data_as(_lib.c_int_p), ext.ctypes.data_as(_lib.c_double_p),
                               65, ptr, ptr, eb.ctypes.data_as(_lib.c_float_p), ptr, None,
                               None, 1e-6, 0.0, 10, it.ctypes.data_as(_lib.c_int_p),
                               stt.ctypes.data_as(_lib.c_int_p), None, None)
    assert rc < 0
    assert b"LSB_NOALLOC_MAX_BATCH" in lib.lsb_last_error()
