"""The allocation-free Hilbert sort (tpm_hilbert_sort_noalloc).

It exists for callers that cannot call cudaMalloc — a simulation whose device
memory all comes from its own pool allocator, or code that must not allocate
in the middle of a stream-ordered pipeline.  The caller owns inputs and
outputs (torch allocates them here, standing in for such a pool); the sort's
intermediate buffers come from the library's fixed device array.  Results
are compared, through the C ABI, with the allocating entry point
(tpm_hilbert_keys) — bit for bit, the tolerance of all integer outputs here —
on two calls in a row, since the shared scratch keeps the previous call's
contents.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _reference(box):
    import treepm
    s = treepm.TreePmSolver(32, box.box_size, 0.0)
    s.set_particles_fixed(box.q, box.mass)
    keys, order = s.hilbert_keys(box.n)
    s.close()
    return keys[order], order


def _noalloc(q, box_size, n_override=None):
    import torch
    from treepm import _lib
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    cols = [torch.from_numpy(np.ascontiguousarray(q[:, a]).view(np.int32)).to(dev) for a in range(3)]
    n = q.shape[0]
    keys = torch.empty(n, dtype=torch.int64, device=dev)
    order = torch.empty(n, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    p = [ctypes.c_void_p(t.data_ptr()) for t in cols]
    rc = lib.tpm_hilbert_sort_noalloc(p[0], p[1], p[2], n if n_override is None else n_override,
                                      float(box_size), ctypes.c_void_p(keys.data_ptr()),
                                      ctypes.c_void_p(order.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc, keys.cpu().numpy().view(np.uint64), order.cpu().numpy().view(np.uint32).astype(np.int64)


def test_noalloc_sort_matches_allocating_entry_point_twice():
    from treepm import ics
    boxes = [ics.clustered_box(24, 200.0, 0.3, 8, min_halo=50, max_halo=500, r_min=0.2, r_max=1.0, seed=91),
             ics.lattice_box(20, 100.0, 1.0, seed=92)]
    for box in boxes:  # two calls in a row, different sizes
        rc, keys, order = _noalloc(box.q, box.box_size)
        assert rc == 0
        ref_keys, ref_order = _reference(box)
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(order, ref_order)


def test_noalloc_sort_at_its_largest_sizes():
    """n = the fixed maximum and one below it: the scratch holds the sort's
    per-tile counts at every accepted size, so both sort bit-exactly."""
    from treepm import _lib, ics
    full = ics.lattice_box(64, 100.0, 1.0, seed=94)
    assert full.n == _lib.NOALLOC_MAX_PARTICLES
    less = ics.Box(full.q[:-1].copy(), full.box_size, full.mass[:-1].copy(), "lattice-1")
    for box in (full, less, full):
        rc, keys, order = _noalloc(box.q, box.box_size)
        assert rc == 0
        ref_keys, ref_order = _reference(box)
        assert np.array_equal(keys, ref_keys)
        assert np.array_equal(order, ref_order)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from treepm import _lib, ics
    box = ics.lattice_box(8, 100.0, 1.0, seed=93)
    rc, _, _ = _noalloc(box.q, box.box_size, n_override=_lib.NOALLOC_MAX_PARTICLES + 1)
    assert rc == 10  # TPM_ERR_TOO_LARGE, nothing launched
