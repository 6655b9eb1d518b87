"""The C-ABI library loads on a machine without a GPU and exports every
function declared in include/*.h."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(sfd_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    from seiscl_b200.engine import load_library

    lib = load_library()
    names = declared_functions()
    assert len(names) >= 15
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_plan_create_without_gpu_fails_cleanly():
    """Without a device the plan cannot be created; the call returns an error
    code instead of crashing."""
    import torch

    from seiscl_b200.engine import Config, Plan, SeisCLEngineError

    if torch.cuda.is_available():
        return
    try:
        Plan(Config(N=[40, 40], ND=2, NT=10, nab=8))
    except SeisCLEngineError as e:
        assert e.code == -2
    else:
        raise AssertionError("plan creation should fail without a CUDA device")


def test_invalid_configs_rejected():
    import ctypes as C

    from seiscl_b200.engine import Config, load_library

    lib = load_library()
    for bad in (dict(N=[41, 40]), dict(N=[40, 40], FDORDER=7), dict(N=[40, 40], MAXRELERROR=5),
                dict(N=[40, 40], ND=5), dict(N=[40, 40], L=9)):
        kw = dict(ND=2, NT=10, nab=8)
        kw.update(bad)
        c = Config(**kw).to_c()
        h = C.c_void_p()
        rc = lib.sfd_plan_create(C.byref(c), C.byref(h))
        assert rc in (-1, -7), bad


def test_fp16_memory_variable_configs():
    """FP16 memory variables under FP32 wave fields: 3D viscoelastic, 8th
    order, NZ a multiple of 4, default kernels, one shot, no checkpointing;
    they halve the memory variables' bytes and nothing else."""
    import dataclasses

    from seiscl_b200.engine import Config, SeisCLEngineError, footprint

    ok = Config(N=[40, 36, 44], ND=3, NT=50, L=2, nab=8, field_precision="fp16_mem")
    f32, f16 = footprint(dataclasses.replace(ok, field_precision="fp32")), footprint(ok)
    assert f32 - f16 == (40 + 8) * (36 + 8) * (44 + 8) * 6 * 2 * 2   # padded cells x 6 variables x L x 2 bytes
    for bad in (dict(ND=2, N=[40, 44]), dict(L=0), dict(FDORDER=4), dict(N=[42, 36, 44]), dict(kernels="general"),
                dict(batch=2), dict(checkpoint=10)):
        with pytest.raises(SeisCLEngineError):
            footprint(dataclasses.replace(ok, **bad))


def test_tma_map_cache_is_thread_safe():
    """The tensor-map cache is read by launches on several threads (the
    service runs plans on worker threads): lookups that evict and rebuild
    entries concurrently must never hand out a torn or stale value."""
    import ctypes as C

    from seiscl_b200.engine import load_library

    lib = load_library()
    fn = lib.sfd_selftest_cache
    fn.restype = C.c_int64
    fn.argtypes = [C.c_int, C.c_int]
    assert fn(8, 20000) == 0
    assert fn(0, 1) < 0
