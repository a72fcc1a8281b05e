"""The allocation-free sample_window entry point (bs_sample_window_static), for callers that cannot allocate
device memory: code under an external memory manager with a fixed budget, or code that must not call
cudaMalloc / cudaFree because those synchronize the device. It takes every array from the caller (here torch
allocates them, as such a caller's own allocator would) and keeps its scratch in one static device array.

Checked through the C ABI against the allocating entry point (bs_sample_window) on two windows in a row, the
second fed with the first's carried samples, bit for bit (the tolerance of every parity test here). This file is
collected last so that a run stopping at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

from ballasim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_static_entry_point_equals_the_allocating_one_on_two_calls(cuda_lib):
    import torch

    from ballasim_b200 import _lib
    from ballasim_b200.sampling import MidpointTest, field_frame, field_levels, field_struct, sample_window

    wl = W.small("blobs", 64, 48, 2)
    spec, r = wl.sensors[0], wl.rules
    f = spec.field
    n = spec.width * spec.height
    ids = np.arange(n, dtype=np.uint32)
    dev = torch.device("cuda")
    blobs_dev = torch.from_numpy(np.ascontiguousarray(f.blobs)).to(dev)
    fs = field_struct(f)
    fs.blobs = blobs_dev.data_ptr()
    rules = _lib.SampleRules(r.tol, r.dark, 1, 1, r.max_refine_levels, r.min_dt_ns, r.l_min, r.l_max)
    mt = MidpointTest(r.tol, r.dark, [1.0], [1.0])
    frame = field_frame(f, 0)

    carried_ref, sig_ref = frame.reshape(n, 1), np.zeros(n, np.uint64)
    ids_d = torch.from_numpy(ids.view(np.int32)).to(dev)
    carried_d = torch.from_numpy(frame.copy()).to(dev)
    sig_d = torch.zeros(n, dtype=torch.int64, device=dev)
    cap = 64 * n
    off_d = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    t_d = torch.zeros(cap, dtype=torch.int64, device=dev)
    irr_d = torch.zeros(cap, dtype=torch.float32, device=dev)
    for w in range(2):  # two calls in a row: the second starts from the first's carried samples
        t_w = w << 23
        lv = field_levels(f, t_w, r.l_min, r.l_max)
        want = sample_window(t_w, ids, lv, ids, carried_ref, sig_ref, f, refine_signature=True, midpoint=mt,
                             max_refine_levels=r.max_refine_levels, min_dt_ns=r.min_dt_ns)
        lv_d = torch.from_numpy(lv).to(dev)
        c_out = torch.zeros(n, dtype=torch.float32, device=dev)
        s_out = torch.zeros(n, dtype=torch.int64, device=dev)
        total = C.c_size_t()
        torch.cuda.synchronize()
        _lib.check(_lib.lib().bs_sample_window_static(
            C.byref(fs), t_w, ids_d.data_ptr(), lv_d.data_ptr(), n, carried_d.data_ptr(), sig_d.data_ptr(),
            C.byref(rules), off_d.data_ptr(), t_d.data_ptr(), irr_d.data_ptr(), cap, c_out.data_ptr(),
            s_out.data_ptr(), None, C.byref(total)))
        S = total.value
        assert S == len(want.t_ns)
        assert np.array_equal(off_d.cpu().numpy(), want.offsets)
        assert np.array_equal(t_d[:S].cpu().numpy(), want.t_ns)
        assert np.array_equal(irr_d[:S].cpu().numpy().view(np.uint32), want.irradiance.reshape(-1).view(np.uint32))
        assert np.array_equal(c_out.cpu().numpy().view(np.uint32), want.last_irradiance.reshape(-1).view(np.uint32))
        assert np.array_equal(s_out.cpu().numpy().view(np.uint64), want.last_signature)
        carried_ref, sig_ref = want.last_irradiance, want.last_signature
        carried_d, sig_d = c_out, s_out

    # Beyond its stated maximum it refuses with a clear error and touches nothing.
    big = (1 << 20) + 1
    with pytest.raises(ValueError, match="exceed its maximum"):
        _lib.check(_lib.lib().bs_sample_window_static(
            C.byref(fs), 0, ids_d.data_ptr(), ids_d.data_ptr(), big, carried_d.data_ptr(), sig_d.data_ptr(),
            C.byref(rules), off_d.data_ptr(), t_d.data_ptr(), irr_d.data_ptr(), cap, c_out.data_ptr(),
            s_out.data_ptr(), None, C.byref(total)))
