"""Host transfers: upload from pageable and pinned memory, and download through the
library's pinned bounce buffer. Downloads are copied out in chunks of 2^20 doubles, so
the vectors here span several chunks and end in a partial one. The round trip must
return the uploaded values exactly (FP64), or their FP32 rounding (FP32 storage)."""
from __future__ import annotations

import numpy as np
import pytest

import gpuqt_b200 as g

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,nvec,precision", [(3_000_017, 1, g.FP64), (1_048_583, 4, g.FP64),
                                              (2_500_009, 4, g.FP32)])
def test_round_trip_across_chunks(n, nvec, precision):
    rng = np.random.default_rng(n + nvec)
    shape = (nvec, n) if nvec > 1 else (n,)
    re = rng.standard_normal(shape)
    im = rng.standard_normal(shape)
    v = g.Vector.from_host(re, im, nvec=nvec, precision=precision)
    got_re, got_im = v.download()
    if precision == g.FP32:
        re, im = re.astype(np.float32).astype(np.float64), im.astype(np.float32).astype(np.float64)
    np.testing.assert_array_equal(got_re, re)
    np.testing.assert_array_equal(got_im, im)


def test_pinned_upload_then_repeated_downloads():
    import torch

    n = 2_097_152
    rng = np.random.default_rng(5)
    re = torch.from_numpy(rng.standard_normal(n)).pin_memory()
    im = torch.from_numpy(rng.standard_normal(n)).pin_memory()
    v = g.Vector(n)
    for _ in range(3):  # the staging pool and the bounce buffer are reused
        v.upload_ptr(re.data_ptr(), im.data_ptr())
        got_re, got_im = v.download()
        np.testing.assert_array_equal(got_re, re.numpy())
        np.testing.assert_array_equal(got_im, im.numpy())
