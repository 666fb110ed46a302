"""tdfs_count_static: counting with no device allocation, working memory in the
library's fixed per-GPU array.  The same counts as tdfs_count on two calls in
a row (the array keeps the previous call's contents, so the second call checks
that everything that must start at zero is cleared), no change in the GPU's
free memory across a call after the first, and oversize graphs rejected
before any GPU work.  Collected after every other test file, so it also runs
on a device where the other entry points have already allocated and run."""
import gc
import random

import numpy as np
import pytest

from tests.golden.make_golden import random_pattern
from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique

CAPACITY = 5  # TDFS_ERR_CAPACITY


def _device_csr(csr):
    import torch
    rowptr = torch.from_numpy(np.ascontiguousarray(csr.rowptr)).cuda()
    colidx = torch.from_numpy(np.ascontiguousarray(csr.colidx)).cuda()
    labels = None if csr.labels is None else torch.from_numpy(np.ascontiguousarray(csr.labels)).cuda()
    torch.cuda.synchronize()
    return rowptr, colidx, labels


def _static(T, csr, dev, P, options=None):
    rowptr, colidx, labels = dev
    return T.count_static(0, csr.n, csr.nedges, rowptr.data_ptr(), colidx.data_ptr(),
                          None if labels is None else labels.data_ptr(), P, options)


def _cases(T):
    rng = random.Random(29)
    er = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    cl = T.gen_chung_lu(20000, 60000, 2.1, 600, 1).set_labels(4, 2)
    er_pats = [(TRIANGLE, False), (CYCLE4, False), (HOUSE, False), (clique(4), False)]
    er_pats += [(random_pattern(6 + t % 2, 0.4, 4, rng), True) for t in range(3)]
    cl_pats = [(TRIANGLE, False), (clique(4), False), (HOUSE, False), (random_pattern(5, 0.5, 4, rng), True)]
    return [(er, er_pats), (cl, cl_pats)]


@pytest.mark.gpu
def test_static_equals_count_two_calls_in_a_row(T):
    for csr, pats in _cases(T):
        G = T.GraphPreprocessor(csr=csr, labeled=True)
        dev = _device_csr(csr)
        for text, labeled in pats:
            P = T.PatternPreprocessor(text=text, labeled=labeled)
            want = T.count(G, P).count
            first = _static(T, csr, dev, P)
            second = _static(T, csr, dev, P)
            assert first == second == want, (text, labeled, first, second, want)


@pytest.mark.gpu
def test_static_options_and_edge_shards(T):
    csr = T.gen_chung_lu(20000, 60000, 2.1, 600, 1)
    G = T.GraphPreprocessor(csr=csr)
    dev = _device_csr(csr)
    P = T.PatternPreprocessor(text=CYCLE4)
    want = T.count(G, P).count
    for opt in ({"steal": 0}, {"merge_window": -1, "chunk_cap": 64}, {"fixed_stage": -1, "edge_chunk": 8}):
        assert _static(T, csr, dev, P, T.default_options(**opt)) == want, opt
    parts = [_static(T, csr, dev, P, T.default_options(edge_stride=3, edge_phase=r)) for r in range(3)]
    assert sum(parts) == want and min(parts) > 0


@pytest.mark.gpu
def test_static_call_allocates_no_device_memory(T):
    import torch
    csr = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    dev = _device_csr(csr)
    P = T.PatternPreprocessor(text=HOUSE)
    first = _static(T, csr, dev, P)  # the first call on the device sets up
    # graphs of earlier tests freed by the collector mid-call would show up
    # as memory returned: collect them first, and hold the collector off
    gc.collect()
    torch.cuda.synchronize()
    gc.disable()
    try:
        free0, _ = torch.cuda.mem_get_info()
        torch_bytes0 = torch.cuda.memory_allocated()
        again = _static(T, csr, dev, P)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
    finally:
        gc.enable()
    assert again == first
    assert free1 == free0 and torch.cuda.memory_allocated() == torch_bytes0


def test_static_rejects_graphs_beyond_the_array(T):
    """Refused from the sizes alone, before any CUDA call (runs without a GPU:
    the pointers are never dereferenced)."""
    P = T.PatternPreprocessor(text=TRIANGLE)
    fake = 256
    for n, e in ((10_000_000, 1_000), (1_000, 20_000_000)):
        with pytest.raises(T.TdfsError) as ei:
            T.count_static(0, n, e, fake, fake, None, P)
        assert ei.value.code == CAPACITY and "scratch" in str(ei.value)


def test_static_rejects_misaligned_colidx(T):
    """colidx is read with 16-byte vector loads: a pointer off a 16-byte
    boundary (a slice such as colidx + 1) is refused before any CUDA call
    (runs without a GPU: the pointers are never dereferenced)."""
    P = T.PatternPreprocessor(text=TRIANGLE)
    for off in (4, 8, 12):
        with pytest.raises(T.TdfsError) as ei:
            T.count_static(0, 100, 400, 256, 256 + off, None, P)
        assert ei.value.code == 7 and "aligned" in str(ei.value)


@pytest.mark.gpu
def test_static_edge_count_not_multiple_of_four(T):
    """A graph whose E is not a multiple of 4, its colidx in a buffer of
    exactly E ints: the count still equals tdfs_count."""
    import torch
    csr = T.gen_er(1001, 7.0, 3)
    assert csr.nedges % 4 != 0
    dev = _device_csr(csr)
    for text in (TRIANGLE, CYCLE4, HOUSE):
        P = T.PatternPreprocessor(text=text)
        want = T.count(T.GraphPreprocessor(csr=csr), P).count
        assert _static(T, csr, dev, P) == want
    torch.cuda.synchronize()
