"""vfrb_dedisperse_noalloc (fixed device scratch) against vfrb_dedisperse.

Both entry points are called through the C ABI on the same inputs; the
no-alloc call gets no workspace at all.  Two different cases run back to
back through the shared scratch, so stale partial sums from the first call
would show in the second call's statistics; the first case and the size
limit run once per dedispersion kernel variant, since each variant writes
the partial sums with its own time blocking.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(vf):
    lib = vf._lib
    lib.vfrb_dedisperse_noalloc.argtypes = [C.c_void_p, C.POINTER(vf.DdArgs), C.c_void_p]
    lib.vfrb_dedisperse_noalloc.restype = C.c_int
    lib.vfrb_dedisperse_noalloc_scratch_bytes.argtypes = []
    lib.vfrb_dedisperse_noalloc_scratch_bytes.restype = C.c_size_t
    return lib


def _filterbank(torch, O, seed, ndm, nch, nt, dm_max):
    rng = np.random.default_rng(seed)
    dms = np.linspace(0, dm_max, ndm).astype(np.float32)
    off, _ = O.delay_table(dms, 384.0, 0.125, 0.001, nch)
    off = np.ascontiguousarray(off, dtype=np.int32)
    rows = nt + int(off.max())
    fb = (rng.standard_normal((nch, rows)) * 5).astype(np.float32)
    d = ndm // 3
    for c in range(nch):
        fb[c, nt // 2 + off[d, c]] += 8.0
    return off, torch.from_numpy(fb).cuda()


def _run(vf, lib, fn, plan, fb, nt, workspace):
    import torch
    dev = fb.device
    ndm = plan.ndm
    out = torch.full((ndm, nt), float("nan"), dtype=torch.float32, device=dev)
    st = dict(ave=torch.full((ndm,), float("nan"), device=dev), sigma=torch.full((ndm,), float("nan"), device=dev),
              peak=torch.full((ndm,), float("nan"), device=dev),
              frb=torch.full((ndm,), -1, dtype=torch.int32, device=dev),
              argmax=torch.full((ndm,), -1, dtype=torch.int32, device=dev))
    a = vf.DdArgs(fb=fb.data_ptr(), storage=vf.F32, chan_scale=None, uniform_scale=0.0, chan_stride=fb.stride(0),
                  row0=0, row_mask=0xFFFFFFFF, nrows_valid=fb.shape[1], nt_out=nt, out=out.data_ptr(),
                  out_stride=out.stride(0), sigma_out=None,
                  workspace=workspace.data_ptr() if workspace is not None else None,
                  workspace_bytes=workspace.numel() if workspace is not None else 0,
                  ave=st["ave"].data_ptr(), sigma=st["sigma"].data_ptr(), peak=st["peak"].data_ptr(),
                  frb=st["frb"].data_ptr(), argmax=st["argmax"].data_ptr(), d_err=None)
    status = fn(plan._p, C.byref(a), None)
    torch.cuda.synchronize()
    return status, out, st


def _compare(got, want):
    out_g, st_g = got
    out_w, st_w = want
    rms = float(out_w.pow(2).mean().sqrt())
    # same kernels, same inputs: well inside the dedispersion tolerance (3e-5 of the rms)
    assert float((out_g - out_w).abs().max()) <= 3e-5 * rms
    for k in ("ave", "sigma", "peak"):
        assert np.allclose(st_g[k].cpu().numpy(), st_w[k].cpu().numpy(), rtol=1e-5, atol=1e-6 * rms), k
    for k in ("frb", "argmax"):
        assert np.array_equal(st_g[k].cpu().numpy(), st_w[k].cpu().numpy()), k


# every kernel variant writes the partial sums with its own time blocking;
# a variant that does not apply to a plan runs the staged kernel instead
VARIANTS = list(range(1, 8))  # VFRB_DD_STAGED .. VFRB_DD_PAT2


def test_noalloc_matches_dedisperse_two_calls(vf, O):
    import torch
    lib = _bind(vf)
    assert lib.vfrb_dedisperse_noalloc_scratch_bytes() == 4 << 20
    cases = [(1, 96, 256, 3000, 120.0, VARIANTS), (2, 40, 192, 700, 60.0, [0])]
    for seed, ndm, nch, nt, dm_max, variants in cases:
        off, fb = _filterbank(torch, O, seed, ndm, nch, nt, dm_max)
        plan = vf.DedispPlan(off)
        ws = torch.empty(plan.workspace_bytes(nt), dtype=torch.uint8, device="cuda")
        for v in variants:
            plan.set_variant(vf.F32, v)
            st_w, *want = _run(vf, lib, lib.vfrb_dedisperse, plan, fb, nt, ws)
            st_g, *got = _run(vf, lib, lib.vfrb_dedisperse_noalloc, plan, fb, nt, None)
            assert st_w == 0 and st_g == 0, v
            _compare(got, want)
            assert int(got[1]["frb"][ndm // 3]) == 1, v


def test_noalloc_size_limit(vf, O):
    import torch
    lib = _bind(vf)
    limit = lib.vfrb_dedisperse_noalloc_scratch_bytes()
    ndm, nch = 4096, 4
    off = np.zeros((ndm, nch), np.int32)
    plan = vf.DedispPlan(off)
    ntb_fit = limit // (24 * ndm)
    rng = np.random.default_rng(5)
    # largest request that fits runs and agrees; one time block more is refused
    nt = 256 * ntb_fit
    assert plan.workspace_bytes(nt) <= limit
    fb = torch.from_numpy(rng.standard_normal((nch, nt + 256)).astype(np.float32)).cuda()
    ws = torch.empty(plan.workspace_bytes(nt), dtype=torch.uint8, device="cuda")
    for v in VARIANTS:
        plan.set_variant(vf.F32, v)
        st_w, *want = _run(vf, lib, lib.vfrb_dedisperse, plan, fb, nt, ws)
        st_g, *got = _run(vf, lib, lib.vfrb_dedisperse_noalloc, plan, fb, nt, None)
        assert st_w == 0 and st_g == 0, v
        _compare(got, want)
        del want, got
    del ws
    nt2 = nt + 256
    assert plan.workspace_bytes(nt2) > limit
    st_r, out_r, _ = _run(vf, lib, lib.vfrb_dedisperse_noalloc, plan, fb, nt2, None)
    assert st_r == 4  # VFRB_ERR_ARG, nothing launched
    assert bool(torch.isnan(out_r).all())
