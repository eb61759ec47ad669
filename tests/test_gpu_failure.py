"""Device-side failure detection, without a GPU fault.

* The tensor-core GEMM's bounded waits: the TMA producer of the first CTA (pair) is told to stop
  before one pipeline stage, so the MMA issuer waits for data that never comes. With every wait
  limited to a short number of cycles the kernel must give up promptly (every role of the CTA
  pair ends at once, since the abort flag is raised in both CTAs), report the failure through
  the C ABI's status word, and leave the context usable: a normal GEMM right after it is exact.
  Nothing here touches a bad address or traps.
* The status words of the plain device path, the batched form and the serving form are zero
  after sound products (the host path checks its own word before returning).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# About 0.1 s at the B200's 1.9 GHz SM clock (0.2 s even at 1 GHz).
LIMIT_CYCLES = 200_000_000


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    return t


@pytest.mark.parametrize("engine_name", ["GEMM_TENSOR", "GEMM_TENSOR_SINGLE"])
def test_withheld_stage_ends_the_gemm_with_an_error(engine_name, fpc, torch):
    engine = getattr(fpc, engine_name)
    m, n, k = 1024, 512, 1024  # 8 K-steps of 128 bytes per tile
    gen = torch.Generator(device="cuda").manual_seed(11)
    a = torch.randint(0, 256, (m, k), dtype=torch.uint8, device="cuda", generator=gen)
    b = torch.randint(0, 256, (n, k), dtype=torch.uint8, device="cuda", generator=gen)
    d = torch.zeros((m, n), dtype=torch.int32, device="cuda")
    fpc.pipeline_status()  # start from a clear device-wide word
    status, flags, elapsed_ms = fpc.gemm_u8_withheld(a.data_ptr(), b.data_ptr(), d.data_ptr(), m, n, k, engine,
                                                     LIMIT_CYCLES, 3)
    assert status == fpc.ECUDA, fpc.last_error()
    assert flags & fpc.STATUS_GEMM_MASK and not flags & ~fpc.STATUS_GEMM_MASK, hex(flags)
    assert "pipeline wait gave up" in fpc.last_error()
    # one limit (plus the 1 ms abort drain), not a chain of every role's own limit
    assert elapsed_ms < 1500, elapsed_ms
    assert fpc.pipeline_status() != 0  # the device-wide diagnostic word saw it too, and is cleared now
    assert fpc.pipeline_status() == 0
    # the context is still usable: the same GEMM without the withheld stage is exact
    status, flags, _ = fpc.gemm_u8_withheld(a.data_ptr(), b.data_ptr(), d.data_ptr(), m, n, k, engine,
                                            LIMIT_CYCLES, 0xFFFFFFFF)
    assert status == fpc.OK and flags == 0, fpc.last_error()
    torch.cuda.synchronize()
    want = a.cpu().numpy().astype(np.int64) @ b.cpu().numpy().astype(np.int64).T
    assert np.array_equal(d.cpu().numpy().astype(np.int64), want)
    assert fpc.pipeline_status() == 0


def test_withheld_check_rejects_bad_arguments(fpc, torch):
    buf = torch.zeros(1 << 16, dtype=torch.uint8, device="cuda")
    status, _, _ = fpc.gemm_u8_withheld(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 128, 256, 128, fpc.GEMM_SIMT,
                                        LIMIT_CYCLES, 0)
    assert status == fpc.EINVAL and "tensor-core engines" in fpc.last_error()
    status, _, _ = fpc.gemm_u8_withheld(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 128, 256, 128, fpc.GEMM_TENSOR,
                                        0, 0)
    assert status == fpc.EINVAL


def test_device_path_status_word_is_clear_after_sound_products(fpc, inputs, oracle, torch):
    n, limbs = 4096, 48
    q, a, b = inputs.instance(n, limbs, 21, 0)
    with fpc.Plan(n, 32 * limbs, limbs, q) as plan:
        da = torch.from_numpy(a.view(np.int32)).cuda()
        db = torch.from_numpy(b.view(np.int32)).cuda()
        dc = torch.empty_like(da)
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(3):
            plan.run_device(da.data_ptr(), db.data_ptr(), dc.data_ptr(), stream)
        assert plan.status() == 0
        assert np.array_equal(dc.cpu().numpy().view(np.uint32), oracle.kronecker(q, a, b))
        assert np.array_equal(plan.run(a, b), oracle.kronecker(q, a, b))  # the host path checks its own word
        assert plan.status() == 0


def test_batch_status_words_after_a_device_run(fpc, inputs, oracle, torch):
    import ctypes
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    h2d, d2h = 1, 2
    shapes = [(1024, 40), (4096, 17), (2048, 90)]
    points = [(n, l) + inputs.instance(n, l, 300 + i, 0) for i, (n, l) in enumerate(shapes)]
    with fpc.Batch([(n, 32 * l, l, q) for n, l, q, _, _ in points]) as batch:
        for i, (n, l, q, a, b) in enumerate(points):
            da, db, _ = batch.io(i)
            assert cudart.cudaMemcpy(da, a.ctypes.data, a.nbytes, h2d) == 0
            assert cudart.cudaMemcpy(db, b.ctypes.data, b.nbytes, h2d) == 0
        batch.run_device(0)
        flags = batch.status()
        assert flags.shape == (len(points),) and not flags.any(), flags
        for i, (n, l, q, a, b) in enumerate(points):
            c = np.empty_like(a)
            assert cudart.cudaMemcpy(c.ctypes.data, batch.io(i)[2], c.nbytes, d2h) == 0
            assert np.array_equal(c, oracle.kronecker(q, a, b)), i
