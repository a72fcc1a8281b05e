"""The allocation-free sample_window entry point (bs_sample_window_static), for callers that cannot allocate device
memory: code under an external memory manager with a fixed budget, or code that must not call cudaMalloc /
cudaFree because those synchronize the device. It takes every array from the caller (here torch allocates them, as
such a caller's own allocator would) and keeps its scratch in one static device array.

Checked through the C ABI against the allocating entry point bs_sample_window (its runs read back with
bs_sampler_download) on two windows in a row, the second fed with the first's carried samples, bit for bit (the
tolerance of every parity test here); then its refusals: more pixels than its maximum, a level above the rules'
finest, a pixel id outside the field, each followed by a valid call that must still match. This file is collected
last so that a run stopping at the first failure has run every other test first."""
import ctypes as C

import numpy as np
import pytest

from ballasim_b200 import workloads as W

pytestmark = pytest.mark.gpu


def allocating_window(sampler, t_w, ids, lv, carried, sig, rules):
    """bs_sample_window through the C ABI: the runs (offsets, t, irr) and the carried samples it writes back."""
    from ballasim_b200 import _lib

    n = len(ids)
    ci = np.ascontiguousarray(carried, np.float32).copy()
    cs = np.ascontiguousarray(sig, np.uint64).copy()
    total = C.c_size_t()
    _lib.check(_lib.lib().bs_sample_window(sampler.h, t_w, ids.ctypes.data, lv.ctypes.data, n, ci.ctypes.data,
                                           cs.ctypes.data, C.byref(rules), C.byref(total)))
    S = total.value
    off = np.zeros(n + 1, np.int64)
    t = np.zeros(S, np.int64)
    irr = np.zeros(S, np.float32)
    _lib.check(_lib.lib().bs_sampler_download(sampler.h, off.ctypes.data, t.ctypes.data, irr.ctypes.data))
    return off, t, irr, ci, cs


def test_static_entry_point_equals_the_allocating_one_on_two_calls(cuda_lib):
    import torch

    from ballasim_b200 import _lib
    from ballasim_b200.sampling import field_frame, field_levels, field_struct, sampler_for

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
    sampler = sampler_for(f)
    frame = field_frame(f, 0)

    carried_ref, sig_ref = frame.copy(), np.zeros(n, np.uint64)
    ids_d = torch.from_numpy(ids.view(np.int32)).to(dev)
    carried_d = torch.from_numpy(frame.copy()).to(dev)
    sig_d = torch.zeros(n, dtype=torch.int64, device=dev)
    cap = 64 * n
    off_d = torch.zeros(n + 1, dtype=torch.int64, device=dev)
    t_d = torch.zeros(cap, dtype=torch.int64, device=dev)
    irr_d = torch.zeros(cap, dtype=torch.float32, device=dev)
    total = C.c_size_t()

    def static_call(t_w, lv_d, c_in, s_in, c_out, s_out, count=n, ids_ptr=None):
        torch.cuda.synchronize()
        return _lib.lib().bs_sample_window_static(
            C.byref(fs), t_w, ids_ptr or ids_d.data_ptr(), lv_d.data_ptr(), count, c_in.data_ptr(), s_in.data_ptr(),
            C.byref(rules), off_d.data_ptr(), t_d.data_ptr(), irr_d.data_ptr(), cap, c_out.data_ptr(),
            s_out.data_ptr(), None, C.byref(total))

    def check_window(t_w, lv, c_out, s_out, want):
        off, t, irr, ci, cs = want
        S = total.value
        assert S == len(t) > n
        assert np.array_equal(off_d.cpu().numpy(), off)
        assert np.array_equal(t_d[:S].cpu().numpy(), t)
        assert np.array_equal(irr_d[:S].cpu().numpy().view(np.uint32), irr.view(np.uint32))
        assert np.array_equal(c_out.cpu().numpy().view(np.uint32), ci.view(np.uint32))
        assert np.array_equal(s_out.cpu().numpy().view(np.uint64), cs)

    for w in range(2):  # two calls in a row: the second starts from the first's carried samples
        t_w = w << 23
        lv = field_levels(f, t_w, r.l_min, r.l_max)
        want = allocating_window(sampler, t_w, ids, lv, carried_ref, sig_ref, rules)
        lv_d = torch.from_numpy(lv).to(dev)
        c_out = torch.zeros(n, dtype=torch.float32, device=dev)
        s_out = torch.zeros(n, dtype=torch.int64, device=dev)
        _lib.check(static_call(t_w, lv_d, carried_d, sig_d, c_out, s_out))
        check_window(t_w, lv, c_out, s_out, want)
        carried_ref, sig_ref = want[3], want[4]
        carried_d, sig_d = c_out, s_out

    # The refusals, each followed by a valid call that still matches the allocating entry point.
    t_w = 2 << 23
    lv = field_levels(f, t_w, r.l_min, r.l_max)
    want = allocating_window(sampler, t_w, ids, lv, carried_ref, sig_ref, rules)
    lv_d = torch.from_numpy(lv).to(dev)
    c_out = torch.zeros(n, dtype=torch.float32, device=dev)
    s_out = torch.zeros(n, dtype=torch.int64, device=dev)
    max_level = 23 - (r.min_dt_ns.bit_length() - 1)
    bad_level = lv.copy()
    bad_level[n // 2] = max_level + 1
    bad_ids = ids.copy()
    bad_ids[n - 1] = n  # one past the field's last pixel
    bad_ids_d = torch.from_numpy(bad_ids.view(np.int32)).to(dev)
    refusals = [
        (dict(count=(1 << 20) + 1), "exceed its maximum"),
        (dict(lv_d=torch.from_numpy(bad_level).to(dev)), "levels must lie in"),
        (dict(ids_ptr=bad_ids_d.data_ptr()), "pixel id outside the field"),
    ]
    for kw, msg in refusals:
        args = dict(lv_d=lv_d, c_in=carried_d, s_in=sig_d, c_out=c_out, s_out=s_out)
        count = kw.pop("count", n)
        ids_ptr = kw.pop("ids_ptr", None)
        args.update(kw)
        with pytest.raises(ValueError, match=msg):
            _lib.check(static_call(t_w, args["lv_d"], args["c_in"], args["s_in"], args["c_out"], args["s_out"],
                                   count=count, ids_ptr=ids_ptr))
        _lib.check(static_call(t_w, lv_d, carried_d, sig_d, c_out, s_out))
        check_window(t_w, lv, c_out, s_out, want)
