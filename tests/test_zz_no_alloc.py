"""The allocation-free operator entry point against the handle-based one (GPU).

fluid_pp_apply_operator_noalloc serves host applications that cannot let a
plug-in allocate device memory (their engine or framework already owns the
GPU's memory).  It must return what fluid_pp_apply_operator returns for the
same state, on every call, using only caller buffers and its fixed scratch:
the device's free memory, torch's allocator and the library's allocation cache
must not change across its calls.  This file is collected last so a failure
here leaves every other test run.
"""
import ctypes

import numpy as np
import pytest

from fluid_b200 import PressureProjector, _abi, configs

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _free_bytes():
    import torch
    free, _total = torch.cuda.mem_get_info(0)
    return int(free)


def _cache_bytes(L):
    out = ctypes.c_ulonglong(0)
    assert L.fluid_pp_allocation_cache_bytes(0, ctypes.byref(out)) == _abi.OK
    return int(out.value)


@pytest.mark.parametrize("dims,seed", [((32, 32, 32), 1), ((37, 50, 29), 11)])
def test_noalloc_operator_matches_handle_on_two_calls(dims, seed):
    import torch

    s = configs.random_small(*dims, seed=seed)
    pp = PressureProjector(dims, s.h)
    pp.upload_state(s.vof, s.u, s.v, s.w)
    pp.prepare(s.dt)
    label, _, diag = pp.level(0)
    rng = np.random.default_rng(seed)
    p = (rng.normal(size=label.shape) * label).astype(np.float32)
    ref = pp.apply_operator(p)                       # existing entry point
    ref_dot = float(np.dot(p.ravel().astype(np.float64), ref.ravel().astype(np.float64)))

    dev = torch.device("cuda:0")
    label_d = torch.from_numpy(np.ascontiguousarray(label)).to(dev)
    diag_d = torch.from_numpy(np.ascontiguousarray(diag)).to(dev)
    p_d = torch.from_numpy(p).to(dev)
    out_d = torch.empty_like(p_d)
    dot_d = torch.empty(1, dtype=torch.float64, device=dev)
    L = _abi.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    nx, ny, nz = dims

    def call():
        return L.fluid_pp_apply_operator_noalloc(nx, ny, nz, _ptr(label_d), _ptr(diag_d), _ptr(p_d), _ptr(out_d),
                                                 _ptr(dot_d), stream)

    def checked_call():
        out_d.fill_(float("nan"))
        dot_d.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = call()
        torch.cuda.synchronize()
        assert rc == _abi.OK, L.fluid_pp_last_error(None)
        out = out_d.cpu().numpy()
        assert np.linalg.norm(out - ref) <= 1e-6 * np.linalg.norm(ref)
        assert abs(float(dot_d.item()) - ref_dot) <= 1e-6 * abs(ref_dot)

    # The first pass through this sequence may load device code (the driver
    # loads a kernel's module at its first launch, this library's and torch's
    # fill kernel alike), which takes device memory that is not an allocation
    # of the entry point; the memory checks bracket the two calls after it.
    checked_call()
    free0, torch0, cache0 = _free_bytes(), torch.cuda.memory_allocated(0), _cache_bytes(L)
    for _call in range(2):
        checked_call()
    assert _free_bytes() == free0, "device free memory changed across the calls"
    assert torch.cuda.memory_allocated(0) == torch0
    assert _cache_bytes(L) == cache0
    pp.destroy()
