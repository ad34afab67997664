"""p3mg_real_forces_noalloc: real-space pair forces that allocate no GPU memory.

The entry point exists for callers that cannot let a library allocate device
memory -- an engine whose own allocator owns all GPU memory (a library-side
cudaMalloc would synchronise the device and fragment that pool), or a
stepping loop that fixes its memory at start-up.  The caller hands over
device buffers for the inputs and outputs; the cell list lives in a fixed
static array inside the library.  These tests call it through the C ABI on
two systems in a row (the array keeps the first call's contents) and compare
with the context-based p3mg_real_forces.  This file is collected last so that
a run stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10   # relative RMS, as for every FP64 parity test
TOL_FP32 = 1e-5    # FP32 sums in a different order


def _entry(lib):
    f = lib.p3mg_real_forces_noalloc
    vp = ctypes.c_void_p
    f.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int, vp,
                  vp, vp]
    f.restype = ctypes.c_int
    return f


def _rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2)) / np.sqrt(np.sum(b ** 2)))


def _reference(x, y, z, q, L, rcut, alpha, precision):
    with p3mg.Context(1, 16, 3, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        return ctx.real_forces(rcut, alpha)


def _device(torch, arrays):
    return [torch.from_numpy(np.ascontiguousarray(a)).to("cuda") for a in arrays]


def test_noalloc_matches_existing_entry_point_two_calls(gpu):
    import torch
    f = _entry(gpu)
    sysA = p3mg.generate_system(0, 20000, 27.1, seed=21) + (27.1, 3.5, 0.9)
    sysB = p3mg.generate_system(4, 7000, 19.0, seed=22) + (19.0, 3.0, 1.1)
    refs = [_reference(*s[:4], s[4], s[5], s[6], p3mg.FP64) for s in (sysA, sysB)]
    ref32 = _reference(*sysA[:4], sysA[4], sysA[5], sysA[6], p3mg.FP32_MIXED)
    outs = []
    free0 = None
    # the first pass is the per-device set-up call (it looks up the array's
    # device address) and also loads torch's own kernels; memory is measured
    # around the calls after it
    for step, (s, prec) in enumerate(((sysB, p3mg.FP32_MIXED), (sysA, p3mg.FP64), (sysB, p3mg.FP64),
                                      (sysA, p3mg.FP32_MIXED))):
        if step == 1:
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            free0 = torch.cuda.mem_get_info()[0]
        x, y, z, q, L, rcut, alpha = s
        n = len(x)
        dx, dy, dz, dq = _device(torch, (x, y, z, q))
        fr = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        e = torch.zeros(1, dtype=torch.float64, device="cuda")
        st = f(n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), dq.data_ptr(), L, rcut, alpha, prec, fr.data_ptr(),
               e.data_ptr(), None)
        assert st == 0, gpu.p3mg_strerror(st)
        torch.cuda.synchronize()
        if step > 0:
            outs.append((fr.cpu().numpy().reshape(3, n), float(e.item())))
        del dx, dy, dz, dq, fr, e
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    # a device allocation by the three measured calls would show up here
    # (the library's array is 6 MiB; one 2 MiB page of slack)
    assert torch.cuda.mem_get_info()[0] >= free0 - (2 << 20)
    for (fr, e), (fr_ref, e_ref) in zip(outs[:2], refs):
        assert _rel(fr, fr_ref) <= TOL_FP64
        assert abs(e - e_ref) <= TOL_FP64 * abs(e_ref)
    assert _rel(outs[2][0], ref32[0]) <= TOL_FP32
    assert abs(outs[2][1] - ref32[1]) <= TOL_FP32 * abs(ref32[1])


def test_noalloc_rejects_sizes_beyond_its_array(gpu):
    """More particles than the static array holds: P3MG_ERR_NOBUF before any work."""
    f = _entry(gpu)
    max_particles = 131072  # P3MG_NOALLOC_MAX_PARTICLES in include/p3mg.h
    assert f(max_particles + 1, None, None, None, None, 10.0, 3.0, 1.0, p3mg.FP64, None, None, None) == -10
    assert f(-1, None, None, None, None, 10.0, 3.0, 1.0, p3mg.FP64, None, None, None) == -1


def _call(torch, f, s, prec, stream=None):
    x, y, z, q, L, rcut, alpha = s
    n = len(x)
    dx, dy, dz, dq = _device(torch, (x, y, z, q))
    fr = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
    e = torch.zeros(1, dtype=torch.float64, device="cuda")
    if stream is not None:
        stream.wait_stream(torch.cuda.current_stream())
    st = f(n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), dq.data_ptr(), L, rcut, alpha, prec, fr.data_ptr(),
           e.data_ptr(), None if stream is None else stream.cuda_stream)
    assert st == 0, p3mg.load().p3mg_strerror(st)
    torch.cuda.synchronize()
    return fr.cpu().numpy().reshape(3, n), float(e.item())


@pytest.mark.parametrize("system_type", [0, 4])
def test_noalloc_capped_cell_grid(gpu, system_type):
    """L / rcut = 50 would give 50 cells per side; the static array holds 16,
    so the cells are about 3 rcut wide.  The Gaussian system (sigma L/6)
    crowds the central cells past the staging capacity, so the chunked
    candidate path runs too.  Compared with the oracle's real space and with
    the context-based entry point, FP64 and FP32, two calls in a row."""
    import torch
    f = _entry(gpu)
    n, L, rcut, alpha = 131072, 50.8, 1.0, 2.5
    x, y, z, q = p3mg.generate_system(system_type, n, L, seed=31 + system_type)
    s = (x, y, z, q, L, rcut, alpha)
    fr_o, e_o = O.realspace(x, y, z, q, L, rcut, alpha, cells=True)
    # FP32 positions are stored relative to their cell's origin; cells three
    # times wider round them three times more coarsely (about 2e-7), and the
    # closest pairs (about 0.01 apart among 131,072 particles) dominate the
    # RMS force: rounding alone moves it by 6e-6 (uniform) / 1.1e-5 (Gaussian)
    tol32 = 5e-5
    for prec, tol in ((p3mg.FP64, TOL_FP64), (p3mg.FP32_MIXED, tol32)):
        ref = _reference(x, y, z, q, L, rcut, alpha, prec)
        for _ in range(2):
            fr, e = _call(torch, f, s, prec)
            assert _rel(fr, ref[0]) <= tol
            assert _rel(fr, fr_o) <= tol
            assert abs(e - e_o) <= tol * abs(e_o)


def test_noalloc_all_pairs_branch_and_side_stream(gpu):
    """Fewer than 3 cells per side (L < 3 rcut) takes the all-pairs kernel;
    the second system runs the cell path on a non-default stream."""
    import torch
    f = _entry(gpu)
    small = p3mg.generate_system(0, 500, 10.0, seed=41) + (10.0, 4.9, 0.7)
    cells = p3mg.generate_system(0, 9000, 21.0, seed=42) + (21.0, 3.2, 1.0)
    side = torch.cuda.Stream()
    for s in (small, cells):
        fr_o, e_o = O.realspace(*s[:4], s[4], s[5], s[6], cells=False)
        for prec, tol in ((p3mg.FP64, TOL_FP64), (p3mg.FP32_MIXED, TOL_FP32)):
            ref = _reference(*s[:4], s[4], s[5], s[6], prec)
            for stream in (None, side):
                fr, e = _call(torch, f, s, prec, stream)
                assert _rel(fr, ref[0]) <= tol
                assert _rel(fr, fr_o) <= tol
                assert abs(e - e_o) <= tol * abs(e_o)
