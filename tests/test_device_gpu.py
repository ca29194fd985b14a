"""Host <-> device transfer helpers on the GPU: the pinned-staging upload of
large strided arrays (with a dtype cast), the batched download (through
staging, or straight into page-locked arrays) and the page-locked host copy."""
import numpy as np
import pytest
import torch

from slm_b200 import device as D

pytestmark = pytest.mark.gpu

DEV = torch.device("cuda", 0)


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint32])
def test_upload_strided_large(dtype):
    rng = np.random.default_rng(1)
    a = (rng.random((2600, 2100, 2)) * 1e6).astype(dtype)  # the [:, :, 1] slice is strided, > 32 MB as float64
    for src in (a[:, :, 1], np.ascontiguousarray(a[:, :, 0])):
        t = D.upload(src, DEV, ("test", str(dtype)), dtype=dtype)
        torch.cuda.synchronize()
        assert np.array_equal(t.cpu().numpy(), src)


def test_upload_bool_mask_and_small():
    m = np.random.default_rng(2).random((7000, 6000)) < 0.3
    t = D.upload(m, DEV, "mask", dtype=np.uint8)
    s = D.upload(m[:10, :10], DEV, "small", dtype=np.uint8)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy(), m.view(np.uint8))
    assert np.array_equal(s.cpu().numpy(), m[:10, :10].view(np.uint8))


def test_download_many():
    ts = [torch.arange(n, dtype=torch.int64, device=DEV) * k for k, n in ((1, 10), (3, 9_000_001), (7, 1))]
    out = D.download(ts, "test")
    for t, o in zip(ts, out):
        assert np.array_equal(o, t.cpu().numpy())
    out[1][0] = -5  # fresh copies, not views of the staging buffers
    assert D.download(ts, "test")[1][0] == 0


def test_download_pinned_fresh_arrays():
    ts = [torch.arange(n, dtype=dt, device=DEV) for n, dt in ((9_000_001, torch.float64), (5, torch.float32))]
    a = D.download(ts, "test", pinned=True)
    b = D.download(ts, "test", pinned=True)
    for t, x, y in zip(ts, a, b):
        assert np.array_equal(x, t.cpu().numpy()) and np.array_equal(y, x)
        assert torch.from_numpy(x).is_pinned()
    a[0][0] = -5  # each call's arrays are its own
    assert b[0][0] == 0


def test_host_copy_pinned_strided():
    a = np.random.default_rng(3).random((3000, 2000, 2)).astype(np.float32)[:, :, 1]
    c = D.host_copy(a, pinned=True)
    assert np.array_equal(c, a) and c.flags.c_contiguous and torch.from_numpy(c).is_pinned()
