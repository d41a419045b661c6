"""The allocation-free step (nsb_gpu_step_noalloc), called through the C ABI,
against the library's regular step (ns_gpu_step) on the same batch: identical
motor outputs, status and full state, bit for bit, on two calls in a row.

The entry point serves callers that may not allocate device memory when they
step (their device memory belongs to another allocator, or they forbid
allocation once started); its scratch lives in a static device array. This
file is collected last so that a failure here leaves every other test run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_step_matches_regular_step_two_calls(nsb):
    batch = nsb.workloads.parity_mix(brains=12)
    regular = nsb.GpuBatch.from_rows(batch)
    noalloc = nsb.GpuBatch.from_rows(batch)
    seeds = np.arange(batch.brains, dtype=np.uint32) + 5
    regular.reset(seeds)
    noalloc.reset(seeds)
    mask = np.ones(batch.brains, np.uint8)
    mask[3] = 0
    for call in range(2):
        out_r, st_r = regular.step(batch.inputs, mask, 16, batch.gain)
        noalloc.upload(batch.inputs, mask)       # caller-owned device buffers: the batch's own
        noalloc.step_noalloc(noalloc.buffer("input"), noalloc.buffer("mask"), 16, batch.gain,
                             noalloc.buffer("output"), noalloc.buffer("status"))
        out_n, st_n = noalloc.download()
        np.testing.assert_array_equal(out_n, out_r, err_msg=f"call {call} outputs")
        np.testing.assert_array_equal(st_n, st_r, err_msg=f"call {call} status")
        for i in range(batch.brains):
            a, b = regular.dump(i), noalloc.dump(i)
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[1], b[1])
            assert a[2] == b[2]
    # synaptic arrivals are counted by both steps alike
    assert regular.take_events() == noalloc.take_events() > 0
    regular.close()
    noalloc.close()


def test_noalloc_rejects_batches_above_the_scratch_limit(nsb):
    """2,097,152 synapses is the limit; one more is refused with a clear error."""
    W = nsb.workloads
    ng = np.array([[0, -1, 1, 0, 0, 1, 1, -52, 0, 0]] * 2, np.float32)
    edges = 2097153
    sg = np.tile(np.array([[0, 1, 1.0, 1, 1, 0, .5, 100, 0, 0, 0]], np.float32), (edges, 1))
    batch = W.Batch(ng, sg, np.array([0, 2]), np.array([0, edges]), np.array([[1]], np.int32), 1, 8, "big",
                    np.zeros((1, 1), np.float32), 230.0)
    big = nsb.GpuBatch.from_rows(batch)
    big.reset(np.zeros(1, np.uint32))
    with pytest.raises(RuntimeError, match="at most 2097152"):
        big.step_noalloc(big.buffer("input"), big.buffer("mask"), 4, 230.0, big.buffer("output"), big.buffer("status"))
    big.close()
