"""sfd_forward_noalloc: forward modelling for callers that cannot allocate.

A caller whose device memory is fixed in advance -- a serving process that
reserved its budget at start-up, or a host application whose allocator owns
the GPU -- cannot have a shot call cudaMalloc.  sfd_forward_noalloc runs the
shot in a fixed array compiled into the library instead, reading the shot
from the caller's device buffers and writing the seismograms into the
caller's device buffer.  This test calls it through the C ABI twice in a row
and compares each result with sfd_forward (the allocating entry point) within
the forward tolerance of the parity tests, on a 2D P-SV grid and on a small
3D viscoelastic grid (4-cell vectorised kernels, whose 128-bit accesses need
16-byte aligned fields, and TMA kernels, whose tensor maps are built over the
array).  It also checks that the first call in a process commits no more
than the array itself (under lazy module loading the driver loads the array
then), that a later call leaves the device's free memory unchanged, and that
an oversized grid is refused.

Named to be collected last, so a run that stops at the first failure has run
every other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

from tests._cases import engine_config, make_case, rel_l2

FWD_TOL = 2e-5  # the forward tolerance of tests/test_gpu_parity.py


def _bind():
    from seiscl_b200.engine import load_library

    lib = load_library()
    fn = lib.sfd_forward_noalloc
    fp = C.c_void_p
    fn.argtypes = [C.c_void_p, fp, fp, C.c_int, fp, C.c_int, C.c_int, C.POINTER(C.c_int), fp, C.c_void_p]
    fn.restype = C.c_int
    return lib, fn


SCRATCH = 16 << 20   # SFD_NOALLOC_SCRATCH_BYTES
_called = []         # set once the entry point has run in this process


def _run_twice(cuda_device, cfg, model, acq, outs, kernels="fast"):
    import torch

    from seiscl_b200.engine import OUT_NAMES, Plan, source_type_mask

    lib, fn = _bind()
    ec = engine_config(cfg)
    ec.kernels = kernels
    plan = Plan(ec)
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    want = plan.forward(acq["src_pos"], acq["src"], acq["rec_pos"], outs)

    nt = cfg["nt"]
    nrec = acq["rec_pos"].shape[0]
    d_sp = torch.from_numpy(acq["src_pos"]).to(cuda_device)
    d_src = torch.from_numpy(acq["src"]).to(cuda_device)
    d_rp = torch.from_numpy(acq["rec_pos"]).to(cuda_device)
    d_seis = torch.zeros((len(outs), nrec, nt), dtype=torch.float32, device=cuda_device)
    sel = (C.c_int * 10)(*[1 if n in outs else 0 for n in OUT_NAMES])
    mask = source_type_mask(acq["src_pos"])
    torch.cuda.synchronize()

    def call():
        rc = fn(plan.h, d_sp.data_ptr(), d_src.data_ptr(), d_sp.shape[0], d_rp.data_ptr(), nrec, mask, sel,
                d_seis.data_ptr(), None)
        assert rc == 0, lib.sfd_last_error(plan.h).decode()
        return d_seis.cpu().numpy()

    free0 = torch.cuda.mem_get_info()[0]
    first = call()
    free1 = torch.cuda.mem_get_info()[0]
    if not _called:
        # the first call of the process may load the array (lazy loading):
        # it commits the array and the code around it, nothing per shot
        assert free0 - free1 <= SCRATCH + (32 << 20), free0 - free1
        _called.append(True)
    else:
        assert free1 == free0
    second = call()
    free2 = torch.cuda.mem_get_info()[0]
    assert free2 == free1
    slots = [n for n in OUT_NAMES if n in outs]
    for got in (first, second):
        for i, n in enumerate(slots):
            assert np.abs(want[n]).max() > 0
            assert rel_l2(got[i], want[n]) < FWD_TOL, n
    return plan


@pytest.mark.gpu
def test_noalloc_forward_matches_sfd_forward_twice(cuda_device):
    cfg, model, acq = make_case(nd=2, nz=64, nx=72, nt=200, freesurf=1, L=1, src_type=100, nab=12)
    _run_twice(cuda_device, cfg, model, acq, ["vx", "vz", "p"])


@pytest.mark.gpu
@pytest.mark.parametrize("kernels", ["fast", "tma"])
def test_noalloc_forward_3d_matches_sfd_forward_twice(cuda_device, kernels):
    # 3D viscoelastic, nz % 4 == 0 and nab % 4 == 0: the 4-cell vectorised
    # kernels (the default) and the TMA kernels over the array
    cfg, model, acq = make_case(nd=3, nz=32, ny=28, nx=36, nt=120, freesurf=1, L=1, src_type=2, nab=8)
    plan = _run_twice(cuda_device, cfg, model, acq, ["vx", "vz", "p"], kernels=kernels)
    assert plan.kernel_family == ("tma" if kernels == "tma" else "vector")


@pytest.mark.gpu
def test_noalloc_refuses_oversized_grid(cuda_device):
    import torch

    from seiscl_b200.engine import OUT_NAMES, Plan

    lib, fn = _bind()
    cfg, model, acq = make_case(nd=2, nz=1200, nx=1200, nt=4, nab=10)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"])
    d = torch.zeros(64, device=cuda_device)
    sel = (C.c_int * 10)(*[1 if n == "vx" else 0 for n in OUT_NAMES])
    rc = fn(plan.h, d.data_ptr(), d.data_ptr(), 1, d.data_ptr(), 1, 16, sel, d.data_ptr(), None)
    assert rc == -4
    msg = lib.sfd_last_error(plan.h).decode()
    assert "bytes" in msg and str(16 << 20) in msg
