"""negacyclic_run_device_static: the device product that allocates nothing.

It serves callers that cannot allocate device memory once running. cudaFree waits
for the whole device. A framework's allocator may hold nearly all of HBM. A host
process may forbid allocations after start-up. Such a caller makes its plan up front
with external_work = 1 (tables only) and multiplies through this entry point, whose
work space is a fixed 64 MiB array in the library.

The checks, through the C ABI:
* two calls in a row match the existing negacyclic_run_device bit for bit, and the
  oracle too (integer product: tolerance 0);
* the plan's own work-space binding is left as it was;
* a call allocates nothing: the device's free memory is the same before and after a
  synchronized call (once the first call has loaded the kernels);
* device-side errors reach the plan's status word, which is clear after these calls;
* a point too large for the array is refused with a message that says so.

This file is collected last, so a run that stops at the first failure has run
every other test before it.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (N, L, seed): 11.8 MiB and 45.9 MiB of work space
SHAPES = [(4096, 64, 0), (8192, 128, 3)]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available(), "GPU tests need a CUDA device"
    return t


def _device(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).cuda()


@pytest.mark.parametrize("n,limbs,seed", SHAPES)
def test_two_calls_match_run_device(n, limbs, seed, fpc, inputs, oracle, torch):
    q, a1, b1 = inputs.instance(n, limbs, seed, 0)
    _, a2, b2 = inputs.instance(n, limbs, seed, 1)
    with_work = fpc.Plan(n, 32 * limbs, limbs, q)                      # existing entry point
    tables_only = fpc.Plan(n, 32 * limbs, limbs, q, external_work=True)  # no work space of its own
    stream = torch.cuda.current_stream().cuda_stream
    try:
        for call, (a, b) in enumerate(((a1, b1), (a2, b2))):
            da, db = _device(torch, a), _device(torch, b)
            want = torch.full_like(da, -1)
            got = torch.full_like(da, -1)
            with_work.run_device(da.data_ptr(), db.data_ptr(), want.data_ptr(), stream)
            tables_only.run_device_static(da.data_ptr(), db.data_ptr(), got.data_ptr(), stream)
            torch.cuda.synchronize()
            assert torch.equal(got, want), f"call {call + 1}"
            if call == 0:
                expect = oracle.kronecker(q, a, b)
                assert np.array_equal(got.cpu().numpy().view(np.uint32), expect)
        assert fpc.pipeline_status() == 0
        assert tables_only.status() == 0
        # the property this entry point exists for: a call leaves the device's free memory as it was
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        tables_only.run_device_static(da.data_ptr(), db.data_ptr(), got.data_ptr(), stream)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before
        assert torch.equal(got, want)
        # the plan without a work space still has none: the static array was bound only for the call
        with pytest.raises(RuntimeError, match="no work space bound"):
            tables_only.run_device(da.data_ptr(), db.data_ptr(), got.data_ptr(), stream)
    finally:
        with_work.close()
        tables_only.close()


def test_plan_keeps_its_own_work_space(fpc, inputs, torch):
    n, limbs, seed = SHAPES[0]
    q, a, b = inputs.instance(n, limbs, seed, 2)
    plan = fpc.Plan(n, 32 * limbs, limbs, q)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        da, db = _device(torch, a), _device(torch, b)
        first, static, again = (torch.full_like(da, -1) for _ in range(3))
        plan.run_device(da.data_ptr(), db.data_ptr(), first.data_ptr(), stream)
        plan.run_device_static(da.data_ptr(), db.data_ptr(), static.data_ptr(), stream)
        plan.run_device(da.data_ptr(), db.data_ptr(), again.data_ptr(), stream)
        torch.cuda.synchronize()
        assert torch.equal(static, first) and torch.equal(again, first)
    finally:
        plan.close()


def test_too_large_a_point_is_refused(fpc, inputs, torch):
    n, limbs = 16384, 256  # about 181 MiB of work space
    q = inputs.random_modulus(limbs, 7)
    plan = fpc.Plan(n, 32 * limbs, limbs, q, external_work=True)
    try:
        assert plan.work_bytes() > 64 << 20
        buf = torch.zeros((n, limbs), dtype=torch.int32, device="cuda")
        with pytest.raises(RuntimeError, match="static work space holds"):
            plan.run_device_static(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 0)
    finally:
        plan.close()
