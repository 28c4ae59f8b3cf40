"""mph_cell_sort_noalloc: the cell sort for callers that cannot allocate.

Callers whose device memory belongs to another allocator, or that run a loop
where cudaMalloc/cudaFree are not allowed, pass their own device buffers; the
sort scratch is a static device array inside the library.  This checks, through
the C ABI, that two calls in a row give exactly (integers: bit for bit) what the
existing path gives -- mph_create's cell build, read back with mph_get_cells
(CellIndex, per-cell ranges) and mph_get_state (ParticleIndex = the bitonic
permutation of the file order).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import mphexplicit_b200 as M
from mphexplicit_b200 import _native as N
from mphexplicit_b200 import scenes

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _noalloc_sort(sc, stream):
    import torch
    lib = N.load()
    c = M.compute_constants(sc.params, sc.header, sc.dim)
    tot = c.total_cell_count
    xyz = torch.tensor(np.ascontiguousarray(sc.xyz), dtype=torch.float64, device="cuda")
    typ = torch.tensor(sc.type, dtype=torch.int32, device="cuda")
    cell_index = torch.full((sc.n,), -7, dtype=torch.int32, device="cuda")
    cell_particle = torch.full((sc.n,), -7, dtype=torch.int32, device="cuda")
    cell_start = torch.full((2 * tot + 1,), -7, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = lib.mph_cell_sort_noalloc(C.byref(c), C.byref(sc.header), sc.n, _ptr(xyz), _ptr(typ), _ptr(cell_index),
                                   _ptr(cell_particle), _ptr(cell_start), C.c_void_p(stream.cuda_stream))
    assert st == 0, st
    stream.synchronize()
    return tot, cell_index.cpu().numpy(), cell_particle.cpu().numpy(), cell_start.cpu().numpy()


def test_noalloc_cell_sort_matches_existing_path_twice():
    import torch
    stream = torch.cuda.Stream()
    cases = [scenes.dam_break_3d(fluid=(12, 10, 16), box=(30, 10, 24), walls=3, seed=41),
             scenes.droplet_2d(n=30, seed=42)]
    for sc in cases:  # two calls in a row, different sizes: the scratch keeps no stale state
        tot, ci, cp, cs = _noalloc_sort(sc, stream)
        s = M.Solver(sc.params, sc.header, sc.type, sc.xyz, sc.vel, dim=sc.dim)
        cells = s.cells()
        st = s.state()
        s.close()
        assert np.array_equal(ci, cells["cell_index"])
        assert np.array_equal(cp, st["particle_index"])
        assert np.array_equal(cs[:tot], cells["fluid_begin"])
        assert np.array_equal(cs[1:tot + 1], cells["fluid_end"])
        assert np.array_equal(cs[tot:2 * tot], cells["wall_begin"])
        assert np.array_equal(cs[tot + 1:2 * tot + 1], cells["wall_end"])


def test_noalloc_call_allocates_no_device_memory():
    """After a first call on the device (its set-up), further calls change
    neither the device's free memory nor torch's allocations."""
    import torch
    stream = torch.cuda.Stream()
    sc = scenes.dam_break_3d(fluid=(10, 8, 12), box=(24, 8, 18), walls=3, seed=43)
    first = _noalloc_sort(sc, stream)
    lib = N.load()
    c = M.compute_constants(sc.params, sc.header, sc.dim)
    tot = c.total_cell_count
    xyz = torch.tensor(np.ascontiguousarray(sc.xyz), dtype=torch.float64, device="cuda")
    typ = torch.tensor(sc.type, dtype=torch.int32, device="cuda")
    out = [torch.zeros(k, dtype=torch.int32, device="cuda") for k in (sc.n, sc.n, 2 * tot + 1)]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    alloc1 = torch.cuda.memory_allocated()
    for _ in range(3):
        st = lib.mph_cell_sort_noalloc(C.byref(c), C.byref(sc.header), sc.n, _ptr(xyz), _ptr(typ), _ptr(out[0]),
                                       _ptr(out[1]), _ptr(out[2]), C.c_void_p(stream.cuda_stream))
        assert st == 0, st
    stream.synchronize()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free1
    assert torch.cuda.memory_allocated() == alloc1
    assert np.array_equal(out[0].cpu().numpy(), first[1]) and np.array_equal(out[1].cpu().numpy(), first[2])


def test_noalloc_cell_sort_rejects_oversize():
    import torch
    sc = scenes.droplet_2d(n=8)
    c = M.compute_constants(sc.params, sc.header, 2)
    big = 1 << 20  # needs a padded size of 2^21 > the static scratch
    dummy = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = N.load().mph_cell_sort_noalloc(C.byref(c), C.byref(sc.header), big, _ptr(dummy), _ptr(dummy),
                                        _ptr(dummy), _ptr(dummy), _ptr(dummy), None)
    assert st == N.MPH_ERR_CAPACITY
    buf = C.create_string_buffer(256)
    N.load().mph_last_error(None, buf, 256)
    assert b"static scratch" in buf.value
