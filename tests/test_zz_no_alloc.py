"""The allocation-free CFL entry point (nhf_cfl_noalloc).

Some callers of this library cannot allocate device memory after start-up:
a host that reserves its whole HBM budget once (a serving process admitting
flood solves against a fixed budget, a model coupler handing out pre-sized
pools) may not call cudaMalloc per request. nhf_cfl_noalloc lets such a
caller ask for the next time-step candidate of a state it owns, using only
its own input and output buffers and a fixed scratch array compiled into
the library. These tests call it through the C ABI and check it against the
handle-based entry point (nhf_compute_cfl + nhf_get_cfl) bit for bit, on two
calls in a row over two different states, so that the scratch contents kept
from the first call cannot leak into the second.
"""
import ctypes

import numpy as np
import pytest


def _noalloc(lib, engine, stream):
    import torch
    t = engine.t
    ndt = torch.full((1,), -1.0, dtype=torch.float32, device=engine.device)
    arg = torch.full((1,), -1, dtype=torch.int32, device=engine.device)
    rc = lib.nhf_cfl_noalloc(t['topology'].data_ptr(), t['bed'].data_ptr(), t['depth'].data_ptr(),
                             t['length'].data_ptr(), t['q'].data_ptr(), engine.arrays.s_num,
                             engine.params.afa, engine.params.g, stream, ndt.data_ptr(), arg.data_ptr())
    assert rc == 0, lib.nhf_cfl_noalloc_error()
    torch.cuda.synchronize(engine.device)
    return float(ndt.item()), int(arg.item())


@pytest.mark.gpu
def test_noalloc_cfl_matches_the_handle_entry_point_on_two_calls(cuda_available):
    import torch
    from nhflood.native import CudaEngine, library
    from nhflood.plain import PlainRun
    from nhflood.workloads import dambreak
    lib = library()
    run = PlainRun(dambreak(n=160, dx=1.0, duration=60), lambda a, p: CudaEngine(a, p, device='cuda:0'))
    try:
        stream = torch.cuda.current_stream(run.engine.device).cuda_stream
        seen = []
        for call in range(2):
            run.advance()  # a different, flowing state for each call
            run.engine.compute_cfl()
            ndt_ref, arg_ref, _ = run.engine.cfl()
            ndt, arg = _noalloc(lib, run.engine, stream)
            assert np.float32(ndt).view(np.uint32) == np.float32(ndt_ref).view(np.uint32), (call, ndt, ndt_ref)
            assert arg == arg_ref, (call, arg, arg_ref)
            assert 0 < arg < run.engine.arrays.s_num and np.isfinite(ndt)
            seen.append((ndt, arg))
        assert seen[0] != seen[1]
    finally:
        run.close()


@pytest.mark.gpu
def test_noalloc_cfl_without_interior_sides_then_a_flowing_mesh(tmp_path, cuda_available):
    """The empty result (+inf and side 0, solver_compact.py:636-639) on a mesh
    whose sides are all exterior and on a mesh without any side (s_num == 1,
    one block that finds nothing), each against the handle entry point, and
    then a flowing dam break, so that the ticket and the block slots are
    shown to be reset between calls."""
    import torch
    from lockstep import workload_from_case
    from nhflood.native import CudaEngine, library
    from nhflood.plain import PlainRun
    from nhflood.workloads import dambreak
    from scenarios import all_cells_filtered, two_cell_case
    lib = library()
    cases = []
    dc, fc = two_cell_case(tmp_path / 'isolated', [[6, 6]], 10)  # two cells, every side exterior
    cases.append(workload_from_case(dc, fc, 'isolated'))
    dc, fc = all_cells_filtered(tmp_path / 'empty')  # no cell and no side: s_num == 1
    cases.append(workload_from_case(dc, fc, 'empty'))
    cases.append(dambreak(n=96, dx=1.0, duration=30))
    for w in cases:
        run = PlainRun(w, lambda a, p: CudaEngine(a, p, device='cuda:0'))
        try:
            run.advance()
            run.engine.compute_cfl()
            ndt_ref, arg_ref, _ = run.engine.cfl()
            stream = torch.cuda.current_stream(run.engine.device).cuda_stream
            ndt, arg = _noalloc(lib, run.engine, stream)
            assert np.float32(ndt).view(np.uint32) == np.float32(ndt_ref).view(np.uint32), (w.name, ndt, ndt_ref)
            assert arg == arg_ref, (w.name, arg, arg_ref)
            if w.name in ('isolated', 'empty'):
                assert np.isinf(ndt) and ndt > 0 and arg == 0, w.name
            else:
                assert np.isfinite(ndt) and arg > 0
        finally:
            run.close()
    assert cases[1].mesh.s_num == 1


@pytest.mark.gpu
def test_noalloc_cfl_refuses_host_pointers(cuda_available):
    """A host array passed as an input is refused before any launch."""
    from nhflood.native import library
    lib = library()
    host = np.zeros(16, np.float32)
    import torch
    dev = torch.zeros(16, device='cuda:0')
    p = ctypes.c_void_p(dev.data_ptr())
    rc = lib.nhf_cfl_noalloc(p, ctypes.c_void_p(host.ctypes.data), p, p, p, 4, 0.5, 9.81, None, p, p)
    assert rc == -1 and b'bed is not' in lib.nhf_cfl_noalloc_error()


def test_noalloc_cfl_rejects_meshes_beyond_its_fixed_scratch():
    """Checked on the host before any device work (runs without a GPU)."""
    from nhflood.native import library
    lib = library()
    fake = ctypes.c_void_p(256)
    rc = lib.nhf_cfl_noalloc(fake, fake, fake, fake, fake, 67_108_864 + 2, 0.5, 9.81, None, fake, fake)
    assert rc == -1
    assert b'67108864-side limit' in lib.nhf_cfl_noalloc_error()
    rc = lib.nhf_cfl_noalloc(None, fake, fake, fake, fake, 10, 0.5, 9.81, None, fake, fake)
    assert rc == -1 and b'null pointer' in lib.nhf_cfl_noalloc_error()
