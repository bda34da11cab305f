"""The allocation-free entry point ``totem_stem_slices_noalloc`` against the session path.

Some callers cannot allocate device memory (their GPU memory belongs to a host framework's
pool, or cudaMalloc's device-wide synchronisation is unaffordable in their serving loop), so
this entry point keeps its intermediate buffers in a fixed device array inside the library and
takes only caller-owned device inputs and outputs.  Here the caller's buffers are torch tensors;
the transmission stack comes from a session run of the same request.  Two consecutive calls
must both reproduce the session's exit-detector images (w_num = 1, so no gfsf weighting) within
the relative L2 tolerance of the other parity tests.  The file sorts last so that a run that
stops at the first failure has run every other test before it.
"""
import numpy as np
import pytest

from tests.conftest import rel_l2
from totem_b200 import capi, request

pytestmark = pytest.mark.gpu
TOL = 1e-4


def test_noalloc_matches_session_twice(engine_lib):
    import torch
    req = request.build_small_stem(mid_layer=())
    assert req.w_num == 1 and req.gfsf[0] == 1.0
    s = capi.Session(device=0)
    s.upload(req)
    s.run()
    ref, _, _ = s.download()
    ref = ref.reshape(req.aper_num, req.depth)
    tptr = s.transmission_ptr()

    dev = torch.device("cuda", 0)
    probe = torch.from_numpy(np.ascontiguousarray(req.probe.astype(np.complex64))).to(dev)
    prop = torch.from_numpy(np.ascontiguousarray(req.prop.astype(np.complex64))).to(dev)
    masks = torch.from_numpy(np.array([np.fft.ifftshift(a) for a in req.aper], dtype=np.float32)).to(dev)
    items = req.w_num * req.depth
    for _ in range(2):
        out = torch.full((req.aper_num * items,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        capi.stem_slices_noalloc(tptr, req.p_height, req.p_width, req.slices, probe.data_ptr(), req.w_num,
                                 prop.data_ptr(), masks.data_ptr(), req.aper_num, req.height, req.step,
                                 req.beginrow, req.begincol, req.width_red, req.depth, 0, items, out.data_ptr())
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(req.aper_num, items)
        assert np.all(np.isfinite(got))
        for a in range(req.aper_num):
            assert rel_l2(got[a], ref[a]) < TOL, (a, rel_l2(got[a], ref[a]))
    s.close()


def test_noalloc_rejects_oversized_batch(engine_lib):
    import torch
    dev = torch.device("cuda", 0)
    n = 512
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    # 64 probes of 512^2 need 128 MiB of scratch, more than the fixed 32 MiB
    with pytest.raises(capi.TotemError) as e:
        capi.stem_slices_noalloc(buf.data_ptr(), 1024, 1024, 2, buf.data_ptr(), 1, buf.data_ptr(), buf.data_ptr(),
                                 2, n, 8, 0, 0, 8, 64, 0, 64, buf.data_ptr())
    assert e.value.code == capi.ERR_INVALID_ARG
    assert "scratch" in str(e.value)


def test_noalloc_split_calls_on_one_stream_with_defocus_spread(engine_lib):
    # A scan cut into consecutive calls (item0 > 0), issued back to back on one caller stream,
    # with three defocus-spread probes (items = w_num * depth): sum_w gfsf_w * result[:, w*depth + pos]
    # must reproduce the session's exit-detector images.
    import torch
    req = request.build_small_stem(raster=(3, 4), focal_steps=3, mid_layer=())
    assert req.w_num == 3
    s = capi.Session(device=0)
    s.upload(req)
    s.run()
    ref, _, _ = s.download()
    ref = ref.reshape(req.aper_num, req.depth)
    tptr = s.transmission_ptr()
    dev = torch.device("cuda", 0)
    probe = torch.from_numpy(np.ascontiguousarray(req.probe.astype(np.complex64))).to(dev)
    prop = torch.from_numpy(np.ascontiguousarray(req.prop.astype(np.complex64))).to(dev)
    masks = torch.from_numpy(np.array([np.fft.ifftshift(a) for a in req.aper], dtype=np.float32)).to(dev)
    items = req.w_num * req.depth
    cuts = [0, 5, 17, items]  # uneven pieces, each crossing probe boundaries
    outs = [torch.full((req.aper_num * (b - a),), float("nan"), dtype=torch.float64, device=dev)
            for a, b in zip(cuts[:-1], cuts[1:])]
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.synchronize()
    for (a, b), out in zip(zip(cuts[:-1], cuts[1:]), outs):
        capi.stem_slices_noalloc(tptr, req.p_height, req.p_width, req.slices, probe.data_ptr(), req.w_num,
                                 prop.data_ptr(), masks.data_ptr(), req.aper_num, req.height, req.step,
                                 req.beginrow, req.begincol, req.width_red, req.depth, a, b - a, out.data_ptr(),
                                 stream.cuda_stream)
    stream.synchronize()
    per_item = np.concatenate([o.cpu().numpy().reshape(req.aper_num, -1) for o in outs], axis=1)
    assert per_item.shape == (req.aper_num, items) and np.all(np.isfinite(per_item))
    got = sum(req.gfsf[w] * per_item[:, w * req.depth:(w + 1) * req.depth] for w in range(req.w_num))
    for a in range(req.aper_num):
        assert rel_l2(got[a], ref[a]) < TOL, (a, rel_l2(got[a], ref[a]))
    s.close()
