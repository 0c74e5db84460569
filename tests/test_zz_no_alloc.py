"""GPU test of gpe_norm_noalloc, the entry point for callers that cannot
allocate device memory where they need a norm (a latency-critical loop that
must not take cudaMalloc/cudaFree's implicit synchronisation, or a process
whose device memory belongs to another allocator).  It computes the same
Simpson norm as gpe_calcnorm but keeps its per-row partials in a file-scope
device array, so the caller only passes psi and the output slot.

The test compares two calls in a row against gpe_calcnorm on the same psi,
within the 1e-12 relative tolerance of the operator-level parity tests, and
checks that a grid beyond the array's capacity is refused.  The device
buffers come from torch; the entry point itself allocates nothing.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12


def _psi(shape, mode):
    rng = np.random.default_rng(11)
    nx, ny, nz = shape
    x = np.linspace(-1, 1, nx)[:, None, None]
    y = np.linspace(-1, 1, ny)[None, :, None]
    z = np.linspace(-1, 1, nz)[None, None, :]
    psi = np.exp(-3 * (x * x + 1.5 * y * y + 2 * z * z)) * (1 + 0.1 * rng.standard_normal(shape))
    if mode == 1:
        psi = psi * np.exp(1j * (0.3 * x + 0.2 * y * z))
    return np.ascontiguousarray(psi)


@pytest.mark.parametrize("mode", [0, 1])
def test_norm_noalloc_matches_calcnorm(gpe_lib, mode):
    import torch

    gpe = gpe_lib
    shape, h = (48, 40, 32), (0.25, 0.2, 0.3)
    s = gpe.Solver(gpe.make_params(mode, *shape, *h, 0.005, 0.5, 1.0, 1.5, 4.0))
    psi = _psi(shape, mode)
    s.set_psi(psi)
    ref = s.calcnorm(False)
    s.close()

    dpsi = torch.from_numpy(psi).to("cuda")  # x-major; complex128 is interleaved (re, im)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for k in range(2):  # two calls in a row share the scratch array
        gpe.norm_noalloc(dpsi.data_ptr(), mode, *shape, *h, out.data_ptr() + 8 * k, stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for v in got:
        assert abs(v / ref - 1.0) <= OP_TOL, (v, ref)


def test_norm_noalloc_rejects_oversize_grid(gpe_lib):
    import torch

    gpe = gpe_lib
    buf = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(gpe.GpeError) as e:
        # 1024 x 512 rows exceed the 262144-row scratch; refused before any launch
        gpe.norm_noalloc(buf.data_ptr(), 0, 1024, 512, 8, 0.1, 0.1, 0.1, buf.data_ptr())
    assert e.value.status == 1 and "262144" in str(e.value)
