"""sfd_forward_noalloc: forward modelling for callers that cannot allocate.

A caller whose device memory is fixed in advance -- a serving process that
reserved its budget at start-up, or a host application whose allocator owns
the GPU -- cannot have a shot call cudaMalloc.  sfd_forward_noalloc runs the
shot in a fixed array compiled into the library instead, reading the shot
from the caller's device buffers and writing the seismograms into the
caller's device buffer.  This test calls it through the C ABI twice in a row
and compares each result with sfd_forward (the allocating entry point) within
the forward tolerance of the parity tests; it also checks that a call leaves
the device's free memory unchanged and that an oversized grid is refused.

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


@pytest.mark.gpu
def test_noalloc_forward_matches_sfd_forward_twice(cuda_device):
    import torch

    from seiscl_b200.engine import OUT_NAMES, Plan, source_type_mask

    lib, fn = _bind()
    cfg, model, acq = make_case(nd=2, nz=64, nx=72, nt=200, freesurf=1, L=1, src_type=100, nab=12)
    plan = Plan(engine_config(cfg))
    plan.set_model(model["vp"], model["vs"], model["rho"], model["taup"], model["taus"])
    outs = ["vx", "vz", "p"]
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

    first = call()
    free_before = torch.cuda.mem_get_info()[0]
    second = call()
    free_after = torch.cuda.mem_get_info()[0]
    assert free_after == free_before
    slots = [n for n in OUT_NAMES if n in outs]
    for got in (first, second):
        for i, n in enumerate(slots):
            assert np.abs(want[n]).max() > 0
            assert rel_l2(got[i], want[n]) < FWD_TOL, n


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
