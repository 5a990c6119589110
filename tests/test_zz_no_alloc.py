"""tk_matvec_host_noalloc: tk_matvec_host staged in the library's static
device array instead of memory allocated per call, for callers that reserve
their device memory up front or cannot pay for cudaMalloc / cudaFree on a
latency-bound path.  Collected last, so it also runs after every other test
has used the library in the same process."""
import numpy as np
import pytest

from conftest import rng
from py_oracle import Q


def jobs(seed, k, n):
    r = rng(seed)
    A = r.integers(0, Q, size=(n, k, k, 256)).astype(np.int16)
    s = r.integers(0, Q, size=(n, k, 256)).astype(np.int16)
    e = r.integers(-3, 4, size=(n, k, 256)).astype(np.int16)
    return A, s, e


def test_rejects_lists_above_the_static_scratch(tk):
    """Checked before any device work (no GPU needed)."""
    k, n = 4, 300                       # 300 * 14 KiB > 4 MiB
    A, s, e = jobs(1, k, n)
    with pytest.raises(tk.TKError) as ex:
        tk.matvec_host_noalloc([(k, A, s, e, np.zeros_like(s))])
    assert ex.value.status == 3 and "static scratch" in str(ex.value)


@pytest.mark.gpu
def test_two_calls_in_a_row_match_matvec_host(tk, cuda):
    import torch
    stream = torch.cuda.Stream()
    for call in range(2):
        items, ref = [], []
        for k, n in ((2, 17), (3, 40), (4, 64)):
            A, s, e = jobs(100 * call + k, k, n)
            items.append((k, A, s, e, np.zeros_like(s)))
            ref.append((k, A, s, e, np.zeros_like(s)))
        tk.matvec_host_noalloc(items, stream=stream)
        tk.matvec_host(ref)
        for a, b in zip(items, ref):
            assert (a[4] == b[4]).all(), call
    assert tk.device_status(0) == 0
