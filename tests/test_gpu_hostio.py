"""Host I/O boundary (orbx_upload_image, orbx_download_points): pitch
conversion with zero padding from pageable and pinned host memory, detection
on an uploaded image, and field-selective keypoint export that leaves the
other fields of each host OrbPoint untouched (the reference's strided copies,
orb.cpp:95-100 and 108-111)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import orbx  # noqa: E402
import synth  # noqa: E402

PT = orbx.ORB_POINT_DTYPE


@pytest.fixture(scope="module")
def ctx():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    c = orbx.Context(0, orbx.make_params(max_pts=10000))
    yield c
    c.close()


def _host_image(w, h, h_pitch, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    img = rng.integers(0, 256, size=(h, h_pitch), dtype=np.uint8)  # padding holds garbage
    return img


@pytest.mark.parametrize("pinned", [False, True])
def test_upload_pitch_conversion(ctx, pinned):
    w, h, hp, dp = 333, 257, 401, 384
    imgs = [_host_image(w, h, hp, s) for s in (1, 2, 3)]
    outs = [torch.full((h, dp), 0xAB, dtype=torch.uint8, device="cuda") for _ in imgs]
    srcs = [torch.from_numpy(x).pin_memory() if pinned else x for x in imgs]
    for src, out in zip(srcs, outs):  # three in a row: the staging buffers alternate
        ctx.upload_image(src, w, h, hp, out, dp)
    ctx.sync()
    for img, out in zip(imgs, outs):
        o = out.cpu().numpy()
        assert np.array_equal(o[:, :w], img[:, :w])
        assert not o[:, w:].any()


def test_detect_on_uploaded_image(ctx):
    a, _, _ = synth.make_pair(640, 480, seed=41)  # (480, 640) with the 128-aligned pitch
    w, h = 640, 480
    # the same picture with a wider, garbage-padded host pitch
    hp = 700
    host = np.full((h, hp), 0x5A, dtype=np.uint8)
    host[:, :w] = a[:, :w]
    d_up = torch.empty((h, a.shape[1]), dtype=torch.uint8, device="cuda")
    ctx.upload_image(host, w, h, hp, d_up, a.shape[1])
    ref = orbx.detect_and_compute(ctx, torch.from_numpy(a).cuda(), w, h)
    ctx.sync()
    rp, rd = ref.to_host()
    got = orbx.detect_and_compute(ctx, d_up, w, h)
    ctx.sync()
    gp, gd = got.to_host()
    assert len(rp) > 100
    assert np.array_equal(rp, gp) and np.array_equal(rd, gd)


@pytest.mark.parametrize("fields", [orbx.FIELDS_KEYPOINT, orbx.FIELDS_MATCH, 3])
def test_download_fields(ctx, fields):
    n = 9973
    rng = np.random.Generator(np.random.PCG64(fields))
    dev_np = np.zeros(n, dtype=PT)
    for f in PT.names:
        dev_np[f] = rng.integers(-1000, 1000, n).astype(PT[f])
    d = torch.from_numpy(dev_np.view(np.int32).reshape(n, 7).copy()).cuda()
    host = np.zeros(n + 5, dtype=PT)
    for f in PT.names:
        host[f] = 77
    ctx.download_points(d, n, host, fields)
    kp = ("x", "y", "octave", "score", "angle")
    mt = ("match", "distance")
    for f in PT.names:
        copied = (f in kp and fields & 1) or (f in mt and fields & 2)
        if copied:
            assert np.array_equal(host[f][:n], dev_np[f]), f
        else:
            assert np.all(host[f][:n] == 77), f
        assert np.all(host[f][n:] == 77)


@pytest.mark.parametrize("with_desc", [False, True])
def test_pair_host_equals_device_pair(ctx, with_desc):
    a, b, _ = synth.make_pair(1920, 1080, seed=43)
    w, h, pitch = 1920, 1080, a.shape[1]
    A, B = orbx.FrameBuffers(10000), orbx.FrameBuffers(10000)
    ctx.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, pitch, A.points, A.desc, A.count,
                 B.points, B.desc, B.count)
    ctx.sync()
    pa, da = A.to_host()
    pb, db = B.to_host()
    for _ in range(2):  # twice: the mapped result block is reused
        hpa = np.full((10000, 7), -7, dtype=np.int32)
        hpb = np.full((10000, 7), -7, dtype=np.int32)
        hna, hnb = np.zeros(1, np.int32), np.zeros(1, np.int32)
        hda = np.zeros((10000, 32), np.uint8) if with_desc else None
        hdb = np.zeros((10000, 32), np.uint8) if with_desc else None
        ctx.pair_host(np.ascontiguousarray(a), np.ascontiguousarray(b), w, h, pitch, hpa, hna, hpb, hnb, hda, hdb)
        assert int(hna[0]) == len(pa) and int(hnb[0]) == len(pb)
        assert np.array_equal(hpa[:len(pa)].view(PT).reshape(-1), pa)
        assert np.array_equal(hpb[:len(pb)].view(PT).reshape(-1), pb)
        assert np.all(hpa[len(pa):] == -7)
        if with_desc:
            assert np.array_equal(hda[:len(pa)], da) and np.array_equal(hdb[:len(pb)], db)


@pytest.mark.parametrize("bands,rows,streams", [(1, 0, 0), (4, 0, 0), (7, 0, 0), (16, 0, 0), (4, 1, 0), (16, 1, 0),
                                                (0, 0, 1)])
@pytest.mark.parametrize("w,h,seed", [(1920, 1080, 44), (333, 257, 45)])
def test_pair_host_overlapped_upload_equals_device_pair(w, h, seed, bands, rows, streams):
    """orbx_pair_host with the images copied in row bands on a second stream,
    while one persistent launch processes the bands that have arrived: the same
    results as orbx_pair on device-resident images, on repeated calls."""
    a, b, _ = synth.make_pair(w, h, seed=seed)
    pitch = a.shape[1]
    ref = orbx.Context(0, orbx.make_params(max_pts=10000))
    A, B = orbx.FrameBuffers(10000), orbx.FrameBuffers(10000)
    ref.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, pitch, A.points, A.desc, A.count,
                 B.points, B.desc, B.count)
    ref.sync()
    pa, da = A.to_host()
    pb, db = B.to_host()
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    t = ctx.get_tuning()
    t.upload_bands = bands
    t.persist_row_deps = rows
    t.host_overlap = streams
    ctx.set_tuning(t)
    ha, hb = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
    for _ in range(3):
        hpa = np.full((10000, 7), -7, dtype=np.int32)
        hpb = np.full((10000, 7), -7, dtype=np.int32)
        hna, hnb = np.zeros(1, np.int32), np.zeros(1, np.int32)
        hda = np.zeros((10000, 32), np.uint8)
        hdb = np.zeros((10000, 32), np.uint8)
        ctx.pair_host(ha.data_ptr(), hb.data_ptr(), w, h, pitch, hpa, hna, hpb, hnb, hda, hdb)
        assert int(hna[0]) == len(pa) and int(hnb[0]) == len(pb)
        assert np.array_equal(hpa[:len(pa)].view(PT).reshape(-1), pa)
        assert np.array_equal(hpb[:len(pb)].view(PT).reshape(-1), pb)
        assert np.array_equal(hda[:len(pa)], da) and np.array_equal(hdb[:len(pb)], db)
    ctx.close()
    ref.close()


@pytest.mark.parametrize("bands,streams", [(0, 0), (4, 0), (0, 1)])
def test_profile_pair_host_phases(bands, streams):
    """orbx_profile_pair_host returns the same results as orbx_pair_host and
    phase times in order: uploads end before the kernels, the kernels before
    the export, and the host wall time covers the device span."""
    w, h = 1920, 1080
    a, b, _ = synth.make_pair(w, h, seed=46)
    pitch = a.shape[1]
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    t = ctx.get_tuning()
    t.upload_bands = bands
    t.host_overlap = streams
    ctx.set_tuning(t)
    ha, hb = torch.from_numpy(a).pin_memory(), torch.from_numpy(b).pin_memory()
    hpa, hpb = np.zeros((10000, 7), np.int32), np.zeros((10000, 7), np.int32)
    hna, hnb = np.zeros(1, np.int32), np.zeros(1, np.int32)
    ctx.pair_host(ha.data_ptr(), hb.data_ptr(), w, h, pitch, hpa, hna, hpb, hnb)
    want = (hpa[:int(hna[0])].copy(), hpb[:int(hnb[0])].copy())
    for _ in range(3):
        ph = ctx.profile_pair_host(ha.data_ptr(), hb.data_ptr(), w, h, pitch, hpa, hna, hpb, hnb)
        assert np.array_equal(hpa[:int(hna[0])], want[0]) and np.array_equal(hpb[:int(hnb[0])], want[1])
        assert 0 < ph["upload_end"] <= ph["kernels_end"] + 1e-3 <= ph["export_end"] + 2e-3
        assert ph["host_wall"] >= ph["export_end"] * 0.9
        assert min(ph[k] for k in ("host_enqueue", "host_wait", "host_copy_out")) >= 0
    ctx.close()


def test_pair_host_graph_follows_contents_and_addresses():
    """orbx_pair_host on two streams replays one captured CUDA graph while the
    pinned images keep their addresses.  New contents at the same addresses
    must be read by the replay, and new addresses must give a new graph: each
    call equals orbx_pair on the same images."""
    w, h = 1280, 720
    imgs = [synth.make_pair(w, h, seed=s)[:2] for s in (60, 61, 62)]
    pitch = imgs[0][0].shape[1]
    ref = orbx.Context(0, orbx.make_params(max_pts=10000))
    want = []
    for a, b in imgs:
        A, B = orbx.FrameBuffers(10000), orbx.FrameBuffers(10000)
        ref.pair_ptr(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(), w, h, pitch, A.points, A.desc, A.count,
                     B.points, B.desc, B.count)
        ref.sync()
        want.append(A.to_host() + B.to_host())
    ref.close()
    ctx = orbx.Context(0, orbx.make_params(max_pts=10000))
    t = ctx.get_tuning()
    t.upload_bands = 0
    t.host_overlap = 1
    ctx.set_tuning(t)
    buf1 = [torch.empty((h, pitch), dtype=torch.uint8).pin_memory() for _ in range(2)]
    buf2 = [torch.empty((h, pitch), dtype=torch.uint8).pin_memory() for _ in range(2)]
    # (image set, buffers): replay, new contents at the same addresses, new addresses, back
    for k, bufs in ((0, buf1), (0, buf1), (1, buf1), (2, buf2), (1, buf1)):
        for dst, src in zip(bufs, imgs[k]):
            dst.copy_(torch.from_numpy(src))
        hpa, hpb = np.full((10000, 7), -7, np.int32), np.full((10000, 7), -7, np.int32)
        hna, hnb = np.zeros(1, np.int32), np.zeros(1, np.int32)
        hda, hdb = np.zeros((10000, 32), np.uint8), np.zeros((10000, 32), np.uint8)
        ctx.pair_host(bufs[0].data_ptr(), bufs[1].data_ptr(), w, h, pitch, hpa, hna, hpb, hnb, hda, hdb)
        pa, da, pb, db = want[k]
        assert int(hna[0]) == len(pa) and int(hnb[0]) == len(pb), k
        assert np.array_equal(hpa[:len(pa)].view(PT).reshape(-1), pa), k
        assert np.array_equal(hpb[:len(pb)].view(PT).reshape(-1), pb), k
        assert np.array_equal(hda[:len(pa)], da) and np.array_equal(hdb[:len(pb)], db), k
    ctx.close()
