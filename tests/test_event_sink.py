"""The event file sink (RawWriter / DatWriter of src/export/raw_writer.h) against the reference's own writers,
compiled from their sources into the harness: the reference pinned to its golden words first (the R-FMT events of
tests/cpp/export/test_export_raw.cpp:170-198), then this build's files byte for byte, with their SHA-256 and stream
counters, over the formats, the TIME_HIGH policies, batch splits, gaps, the 2^28-step wrap and the refusals. The
header-only cases (no events) and the SHA-256 run on the CPU; the words are built on the device (gpu cases)."""
import hashlib
import zlib

import numpy as np
import pytest

FORMATS = ["evt2", "evt2_change", "evt21", "evt3", "dat"]


def _golden():
    """R-FMT's seven events (u in us, each at t_ns = 1000 u + 419)."""
    u = np.array([0, 0, 0, 1, 64, 4096, 4097], np.int64)
    x = np.array([10, 11, 12, 639, 3, 3, 1279], np.uint16)
    y = np.array([5, 5, 5, 479, 0, 0, 719], np.uint16)
    p = np.array([1, 1, 1, 0, 1, 0, 1], np.uint8)
    return x, y, p, 1000 * u + 419


def _th32(step):
    return "%08x" % (0x80000000 | (step & 0x0FFFFFFF))


GOLDEN_EVT2_HEAD = ["80000000", "10005005", "10005805", "10006005", "0053f9df", "80000000", "80000000", "80000000",
                    "80000001", "10001800"]
GOLDEN_EVT2_TAIL = ["80000040", "00001800", "1067facf"]
GOLDEN_EVT2_CHANGE = ["80000000", "10005005", "10005805", "10006005", "0053f9df", "80000001", "10001800",
                      "80000040", "00001800", "1067facf"]
GOLDEN_EVT21 = ["8000000000000000", "1000000500001c00", "005301df80000000", "8000000100000000", "1000000000000008",
                "8000004000000000", "0000000000000008", "106702cf80000000"]
GOLDEN_EVT3 = ["8000", "6000", "0005", "280a", "280b", "280c", "6001", "01df", "227f", "6040", "0000", "2803", "8001",
               "6000", "2003", "6001", "02cf", "2cff"]
GOLDEN_DAT = ("000000000a400110000000000b400110000000000c400110010000007fc277004000000003000010001000000300000001100000"
              "ffc4b310")


def _words(data: bytes, size: int):
    body = data[data.index(b"% end\n") + 6:]
    assert len(body) % size == 0
    return ["%0*x" % (2 * size, int.from_bytes(body[i:i + size], "little")) for i in range(0, len(body), size)]


def _check_golden(data: dict):
    ob = _words(data["evt2"], 4)
    assert len(ob) == 264
    assert ob[:10] == GOLDEN_EVT2_HEAD and ob[-3:] == GOLDEN_EVT2_TAIL
    assert ob[10:261] == [_th32(1 if i < 13 else 2 + (i - 13) // 4) for i in range(10, 261)]
    assert _words(data["evt2_change"], 4) == GOLDEN_EVT2_CHANGE
    assert _words(data["evt21"], 8) == GOLDEN_EVT21
    assert _words(data["evt3"], 2) == GOLDEN_EVT3
    dat = data["dat"]
    assert dat[dat.index(b"\x0c\x08") + 2:].hex() == GOLDEN_DAT


def _fmt(name):
    """(format, evt2_time_high) of a case name."""
    return ("evt2", "change") if name == "evt2_change" else (name, "openeb")


def _ref_file(ref, path, name, cols, bounds=None, width=1280, height=720, origin_us=0, epoch_ns=0, rem=(419, 419),
              version="0.0.0"):
    fmt, th = _fmt(name)
    info, refused, msg = ref.event_file(path, fmt, width, height, origin_us, epoch_ns, *cols, bounds=bounds,
                                        evt2_time_high=th, t_ns_rem_min=rem[0], t_ns_rem_max=rem[1], version=version)
    return path.read_bytes(), info, refused, msg


def _our_writer(path, name, width=1280, height=720, origin_us=0, epoch_ns=0, rem=(419, 419), version="0.0.0"):
    from ballasim_b200.export import DatWriter, RawWriter

    fmt, th = _fmt(name)
    if fmt == "dat":
        return DatWriter(str(path), width, height, origin_us, epoch_ns, rem[0], rem[1], version)
    return RawWriter(str(path), fmt, width, height, origin_us, epoch_ns, th, rem[0], rem[1], version)


def _our_file(path, name, cols, bounds=None, **kw):
    from ballasim_b200.export import ExportError

    w = _our_writer(path, name, **kw)
    x, y, p, t = cols
    b = [0, len(t)] if bounds is None else list(bounds)
    refused, msg = [], ""
    for a, e in zip(b[:-1], b[1:]):
        try:
            w.append(x[a:e].copy(), y[a:e].copy(), p[a:e].copy(), t[a:e].copy())
            refused.append(False)
        except ExportError as err:
            refused.append(True)
            msg = str(err)
    info = w.close()
    assert info["path"] == str(path)
    return path.read_bytes(), info, np.array(refused, bool), msg


def _same(ours, theirs):
    data, info, refused, msg = ours
    r_data, r_info, r_refused, r_msg = theirs
    assert data == r_data
    assert info["bytes"] == r_info["bytes"] == len(data)
    assert info["sha256"] == r_info["sha256"] == hashlib.sha256(data).hexdigest()
    s = info["streams"][0]
    assert (s["count"], s["t_first"], s["t_last"]) == (r_info["count"], r_info["t_first"], r_info["t_last"])
    assert np.array_equal(refused, r_refused)
    assert msg == r_msg


def test_reference_writers_give_the_golden_words(ref, tmp_path):
    cols = _golden()
    _check_golden({name: _ref_file(ref, tmp_path / f"{name}.raw", name, cols)[0] for name in FORMATS})


def test_sha256_matches_hashlib():
    from ballasim_b200.export import sha256_hex

    rng = np.random.default_rng(5)
    for n in (0, 3, 55, 56, 63, 64, 65, 119, 4096, 100_003):
        d = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert sha256_hex(d) == hashlib.sha256(d).hexdigest()
    assert sha256_hex(b"abc") == "ba7816bf8f01cfea414140de5dae2223b00361a396177a9cb410ff61f20015ad"


@pytest.mark.parametrize("name", FORMATS)
@pytest.mark.parametrize("opts", [
    dict(),
    dict(origin_us=123456, epoch_ns=1_700_000_000_000_000_000, rem=(-1, -1), version=""),
    dict(origin_us=-5, epoch_ns=-86_400_000_000_000 * 365 * 3, rem=(0, 999), version="1.2.3 beta"),
])
def test_headers_of_files_without_events(ref, tmp_path, name, opts):
    """The header (format line, integrator names, plugin_version, the date of epoch + origin, the T1a keys) and the
    closed file's size, hash and empty stream, with no device work."""
    _same(_our_file(tmp_path / "ours", name, _golden(), bounds=[0], **opts),
          _ref_file(ref, tmp_path / "ref", name, _golden(), bounds=[0], **opts))


@pytest.mark.parametrize("kw", [
    dict(width=0), dict(height=2049), dict(epoch_ns=1500), dict(rem=(5, 3)), dict(rem=(-1, 3)), dict(rem=(0, 1000)),
    dict(version="bad\nline"), dict(origin_us=2 ** 62),
])
def test_writer_arguments_are_refused_as_the_reference_refuses_them(ref, tmp_path, kw):
    from ballasim_b200.export import ExportError, RawWriter

    for name in ("evt3", "dat"):
        if name == "dat" and kw.get("height") == 2049:
            continue  # DAT takes 14-bit addresses
        with pytest.raises(ValueError):
            _ref_file(ref, tmp_path / "ref", name, _golden(), bounds=[0], **kw)
        with pytest.raises(ExportError):
            _our_writer(tmp_path / "ours", name, **kw)
    with pytest.raises(ExportError, match="unknown RAW format"):
        RawWriter(str(tmp_path / "x"), "evt4", 8, 8, 0, 0)
    with pytest.raises(ExportError, match="unknown evt2_time_high"):
        RawWriter(str(tmp_path / "x"), "evt2", 8, 8, 0, 0, "sometimes")


def test_append_checks_dtypes_and_lengths_before_any_work(tmp_path):
    from ballasim_b200.export import ExportError

    w = _our_writer(tmp_path / "f", "evt3")
    x, y, p, t = _golden()
    with pytest.raises(TypeError):
        w.append(x.astype(np.int32), y, p, t)
    with pytest.raises(TypeError):
        w.append(x, y, p, t.astype(np.float64))
    with pytest.raises(ExportError, match="one length"):
        w.append(x[:3], y, p, t)
    w.append(x[:0], y[:0], p[:0], t[:0])
    info = w.close()
    assert info["streams"][0]["count"] == 0
    with pytest.raises(ExportError, match="append after close"):
        w.append(x, y, p, t)
    with pytest.raises(ExportError, match="closed twice"):
        w.close()


# ---------------------------------------------------------------------------------------------------------------
# the device encoder
# ---------------------------------------------------------------------------------------------------------------

def _stream(rng, n, width=1280, height=720, t0_us=0, gap_every=0, gap_us=0, rem=419):
    """Events in output order: runs of equal times (EVT 2.1 words of several events, duplicates), y and x runs, idle
    gaps; t_ns = 1000 u + rem."""
    du = rng.choice([0, 0, 0, 1, 2, 17, 64, 300, 5000], n, p=[.3, .1, .1, .2, .1, .08, .06, .04, .02])
    if gap_every:
        du[::gap_every] += gap_us
    u = t0_us + np.cumsum(du)
    y = rng.integers(0, height, n).astype(np.uint16)
    same = rng.random(n) < 0.5
    y[1:][same[1:]] = y[:-1][same[1:]]  # runs of one row
    x = rng.integers(0, width, n).astype(np.uint16)
    step = rng.integers(1, 4, n)
    for i in range(1, n):  # runs of increasing x within a 32-pixel base, and some repeats
        if same[i] and rng.random() < 0.7:
            x[i] = min(width - 1, int(x[i - 1]) + int(step[i]) - (1 if rng.random() < 0.1 else 0))
    p = (rng.random(n) < 0.5).astype(np.uint8)
    p[1:][same[1:]] = p[:-1][same[1:]]
    return x, y, p, (1000 * u + rem).astype(np.int64)


@pytest.mark.gpu
def test_device_encoder_gives_the_golden_words(cuda_lib, tmp_path):
    cols = _golden()
    _check_golden({name: _our_file(tmp_path / f"{name}.raw", name, cols)[0] for name in FORMATS})


@pytest.mark.gpu
@pytest.mark.parametrize("name", FORMATS)
@pytest.mark.parametrize("case", ["one", "batches", "gaps", "wrap"])
def test_files_equal_the_reference_byte_for_byte(cuda_lib, ref, tmp_path, name, case):
    rng = np.random.default_rng(zlib.crc32(f"{name}/{case}".encode()))
    kw = dict(origin_us=1_000, epoch_ns=1_650_000_000_000_000_000)
    if case == "one":
        cols, bounds = _stream(rng, 20_000, t0_us=1_000), None
    elif case == "batches":
        cols = _stream(rng, 200_000, t0_us=1_000)
        cuts = np.unique(np.concatenate([[0, 1, 8, 1005, 131_072], rng.integers(0, 200_000, 20), [200_000]]))
        bounds = cuts
    elif case == "gaps":  # idle gaps of 10 ms to 2 s: keepalives and long TIME_HIGH runs
        cols, bounds = _stream(rng, 5_000, t0_us=1_000, gap_every=97, gap_us=int(rng.integers(10_000, 2_000_000))), \
            [0, 2_000, 2_001, 5_000]
    else:  # across EVT 2.0/2.1's 2^28-step TIME_HIGH wrap (u = 2^34 us) and EVT 3.0's 2^24 us loops
        start = (1 << 34) - 3_000_000 if name != "dat" else (1 << 32) - 3_000_000 - 1_000_000
        cols, bounds = _stream(rng, 30_000, t0_us=start + 1_000, gap_every=11, gap_us=1_000), [0, 10_000, 30_000]
        if name == "dat":
            cols = tuple(c[:2_000] for c in cols)
            bounds = [0, 1_000, 2_000]
    _same(_our_file(tmp_path / "ours", name, cols, bounds, **kw), _ref_file(ref, tmp_path / "ref", name, cols, bounds,
                                                                          **kw))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["evt2_change", "evt21", "evt3"])
def test_hours_long_gaps_across_the_time_high_wrap(cuda_lib, ref, tmp_path, name):
    """Idle gaps of hours: on-change keepalives by the million, the 2^28-step block start (u = 2^34 us) crossed
    inside a gap (EVT 2.1's guard word before a keepalive) and right at an event; EVT 3.0's dense TIME_HIGH."""
    rng = np.random.default_rng(29)
    origin = 1_000
    a = _stream(rng, 3_000, t0_us=origin + (1 << 34) - 5_000_000)
    b = _stream(rng, 3_000, t0_us=origin + (1 << 34) + 3 * 3600 * 1_000_000)  # 3 hours later, past the block start
    c = _stream(rng, 50, t0_us=origin + (1 << 35) - 64 * 128 * 3)  # keepalives, then an event on a block start
    u_single = np.array([(1 << 35), (1 << 35) + (1 << 34) - 64 * 100, (1 << 35) + (1 << 34)], np.int64)
    d = (np.array([5, 6, 7], np.uint16), np.array([7, 7, 7], np.uint16), np.array([1, 0, 1], np.uint8),
         1000 * (origin + u_single) + 419)  # the last: a block start with no keepalive before it
    cols = tuple(np.concatenate(z) for z in zip(a, b, c, d))
    assert np.all(np.diff(cols[3]) >= 0)
    bounds = [0, 3_000, 3_001, 6_000, len(cols[3])]
    kw = dict(origin_us=origin, epoch_ns=0)
    _same(_our_file(tmp_path / "ours", name, cols, bounds, **kw), _ref_file(ref, tmp_path / "ref", name, cols, bounds,
                                                                          **kw))


@pytest.mark.gpu
@pytest.mark.parametrize("name", FORMATS)
def test_refused_batches_write_nothing_and_name_the_reference_reason(cuda_lib, ref, tmp_path, name):
    rng = np.random.default_rng(11)
    x, y, p, t = (c.copy() for c in _stream(rng, 6_000, t0_us=1_000))
    bounds = [0, 1_000, 2_000, 3_000, 4_000, 5_000, 6_000]
    t[1_500] = t[1_499] - 1  # out of order
    x[2_700] = 1280  # outside the sensor
    p[3_100] = 2  # polarity
    t[4_200:] += 1  # sub-us part 420: outside the declared [419, 419] from here on
    t[5_000:] -= 1
    kw = dict(origin_us=1_000, epoch_ns=0)
    ours = _our_file(tmp_path / "ours", name, (x, y, p, t), bounds, **kw)
    theirs = _ref_file(ref, tmp_path / "ref", name, (x, y, p, t), bounds, **kw)
    assert list(ours[2]) == [False, True, True, True, True, False]
    _same(ours, theirs)
    # Events before the origin; EVT 2.0/2.1's first event at u >= 2^34; DAT's u >= 2^32.
    early = (x[:5], y[:5], p[:5], t[:5] - 1_000_000_000)
    _same(_our_file(tmp_path / "o2", name, early, **kw), _ref_file(ref, tmp_path / "r2", name, early, **kw))
    late = (x[:5], y[:5], p[:5], t[:5] + 1000 * ((1 << 34) + 5))
    _same(_our_file(tmp_path / "o3", name, late, **kw), _ref_file(ref, tmp_path / "r3", name, late, **kw))


@pytest.mark.gpu
def test_device_columns_give_the_same_file(cuda_lib, tmp_path):
    """append_device on device columns (the output stage's kind) writes what append writes from the host."""
    import torch

    rng = np.random.default_rng(3)
    cols = _stream(rng, 50_000, t0_us=10)
    a = _our_file(tmp_path / "host", "evt21", cols)[0]
    w = _our_writer(tmp_path / "dev", "evt21")
    d = [torch.from_numpy(c.view(np.int16) if c.dtype == np.uint16 else c).cuda() for c in cols]
    torch.cuda.synchronize()
    w.append_device(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), len(cols[3]))
    w.close()
    assert (tmp_path / "dev").read_bytes() == a
    st = w.stats()
    assert st["gpu_launches"] >= 5 and st["last_kernel_ms"] > 0
    assert st["last_words_bytes"] == len(a) - a.index(b"% end\n") - 6 - 8  # all but the header and the open word
