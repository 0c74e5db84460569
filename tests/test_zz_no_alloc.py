"""Tests of gpe_norm_noalloc, the entry point for callers that cannot
allocate device memory where they need a norm (a latency-critical loop that
must not take cudaMalloc/cudaFree's implicit synchronisation, or a process
whose device memory belongs to another allocator).  It computes the same
Simpson norm as gpe_calcnorm but keeps its per-row partials in a file-scope
device array, so the caller only passes psi and the output slot.

GPU tests: two calls in a row against gpe_calcnorm on the same psi, within
the 1e-12 relative tolerance of the operator-level parity tests, on even grids
including the array's capacity (nx * ny = 262144 with nx = 1024); odd grids
(which the solver handle does not accept) against the Simpson rule with the
reference's weights; and no change of the device's free memory across the
calls.  CPU tests: misaligned pointers and sizes beyond the array are refused
with GPE_ERR_PARAM before anything touches the GPU.  The device buffers come
from torch; the entry point itself allocates nothing.
"""
import numpy as np
import pytest

OP_TOL = 1e-12
GPE_ERR_PARAM = 1


def _psi(shape, mode, seed=11):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x = np.linspace(-1, 1, nx)[:, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None]
    z = np.linspace(-1, 1, nz)[None, None, :]
    psi = np.exp(-3 * (x * x + 1.5 * y * y + 2 * z * z)) * (1 + 0.1 * rng.standard_normal(shape))
    if mode == 1:
        psi = psi * np.exp(1j * (0.3 * x + 0.2 * y * z))
    return np.ascontiguousarray(psi)


def _simpson_weights(n):
    # the composite Simpson rule of simpint (diffint.cu:37-66) as weights
    m = n if n % 2 else n - 1
    w = np.zeros(n)
    w[0:m] = 2.0
    w[1:m:2] = 4.0
    w[0] = w[m - 1] = 1.0
    if n % 2 == 0:
        w[n - 1] += 5 / 4
        w[n - 2] += 8 / 4
        w[n - 3] -= 1 / 4
    return w / 3


def _numpy_norm(psi, h):
    rho = np.abs(psi) ** 2
    for ax in (2, 1, 0):
        rho = h[ax] * np.tensordot(rho, _simpson_weights(psi.shape[ax]), axes=([rho.ndim - 1], [0]))
    return float(np.sqrt(rho))


def _noalloc_twice(gpe, psi, mode, shape, h):
    """Two calls in a row on one stream; returns both norms and the device's
    free memory before and after them."""
    import torch

    dpsi = torch.from_numpy(psi).to("cuda")  # x-major; complex128 is interleaved (re, im)
    out = torch.full((3,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # first call: loads the module holding the array and caches its address
    gpe.norm_noalloc(dpsi.data_ptr(), mode, *shape, *h, out.data_ptr() + 16, stream)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(2):  # two calls in a row share the scratch array
        gpe.norm_noalloc(dpsi.data_ptr(), mode, *shape, *h, out.data_ptr() + 8 * k, stream)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    return out.cpu().numpy()[:2], free0, free1


EVEN = [(48, 40, 32), (1024, 256, 8), (18, 10, 1024)]


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", EVEN)
def test_norm_noalloc_matches_calcnorm(gpe_lib, mode, shape):
    gpe = gpe_lib
    h = (0.25, 0.2, 0.3)
    s = gpe.Solver(gpe.make_params(mode, *shape, *h, 0.005, 0.5, 1.0, 1.5, 4.0))
    psi = _psi(shape, mode)
    s.set_psi(psi)
    ref = s.calcnorm(False)
    s.close()
    got, free0, free1 = _noalloc_twice(gpe, psi, mode, shape, h)
    for v in got:
        assert abs(v / ref - 1.0) <= OP_TOL, (v, ref)
    assert free1 == free0  # nothing was allocated by the two calls


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", [(17, 13, 11), (9, 30, 7)])
def test_norm_noalloc_odd_grids(gpe_lib, mode, shape):
    h = (0.25, 0.2, 0.3)
    psi = _psi(shape, mode, seed=5)
    ref = _numpy_norm(psi, h)
    got, free0, free1 = _noalloc_twice(gpe_lib, psi, mode, shape, h)
    for v in got:
        assert abs(v / ref - 1.0) <= OP_TOL, (v, ref)
    assert free1 == free0


@pytest.mark.parametrize("args, msg", [
    # 1024 x 512 rows exceed the 262144-row scratch
    ((0x1000, 0, 1024, 512, 8), "262144"),
    # a y extent whose product with nx would wrap a 64-bit long
    ((0x1000, 0, 16, 2 ** 62, 8), "262144"),
    ((0x1000, 0, 16, 16, 2048), "nz exceeds"),
    ((0x1000, 0, 2048, 16, 16), "nx exceeds"),
    # complex psi 8 bytes past a 16-byte boundary (an offset view of a buffer)
    ((0x1008, 1, 16, 16, 16), "16-byte aligned"),
    ((0x1004, 0, 16, 16, 16), "8-byte aligned"),
])
def test_norm_noalloc_refuses_before_any_launch(gpe_lib, args, msg):
    """Refusals come from argument checks that run before any CUDA call, so
    these fake device addresses are never dereferenced (no GPU needed)."""
    gpe = gpe_lib
    ptr, mode, nx, ny, nz = args
    with pytest.raises(gpe.GpeError) as e:
        gpe.norm_noalloc(ptr, mode, nx, ny, nz, 0.1, 0.1, 0.1, 0x2000)
    assert e.value.status == GPE_ERR_PARAM and msg in str(e.value)
    with pytest.raises(gpe.GpeError) as e:
        gpe.norm_noalloc(0x1000, 0, 16, 16, 16, 0.1, 0.1, 0.1, 0x2004)  # misaligned output slot
    assert e.value.status == GPE_ERR_PARAM and "norm_dev" in str(e.value)
