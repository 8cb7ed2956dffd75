"""The graph-recorded batch (GLS_GRAPH): frames of uneven sizes give the
same bits as the stream-launched batch, replays read the current contents
of the same buffers, and a change of parameter values records a new graph."""
import numpy as np
import pytest
import torch

from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu

SIZES = [(320, 240), (256, 192), (192, 144), (384, 288)]


def _batch(seed, iso=800):
    raws, params = [], []
    for k, (w, h) in enumerate(SIZES):
        wl = scene.Workload(f"m{k}", w, h, levels=4, gain=1.0 + 0.3 * k, read=3.0 + k, iso=iso, seed=seed + k,
                            white=4095 if k % 2 == 0 else 16383, black=512 if k % 2 == 0 else 2048)
        raw, _ = scene.make_raw(wl)
        raws.append(torch.from_numpy(raw.view(np.int16)).cuda())
        params.append(scene.make_params(wl))
    return raws, params


def _outs():
    return [torch.empty((h, w, 4), dtype=torch.float16, device="cuda") for (w, h) in SIZES]


def test_graph_batch_matches_stream_batch(converter):
    st = torch.cuda.Stream()
    raws, params = _batch(100)
    ref, got = _outs(), _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    converter.demosaic_batch(raws, params, got, stream=st, graph=True)  # runs and records
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))
    for o in got:
        o.zero_()
    converter.demosaic_batch(raws, params, got, stream=st, graph=True)  # replays
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))


def test_graph_replay_reads_new_contents_and_rerecords_on_new_params(converter):
    st = torch.cuda.Stream()
    raws, params = _batch(200)
    got = _outs()
    converter.demosaic_batch(raws, params, got, stream=st, graph=True)
    new_raws, _ = _batch(300)
    for r, n in zip(raws, new_raws):
        r.copy_(n)  # same buffers, new frames
    ref = _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    converter.demosaic_batch(raws, params, got, stream=st, graph=True)
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))
    _, p2 = _batch(200, iso=1600)  # other parameter values: a new recording
    converter.demosaic_batch(raws, p2, ref, stream=st)
    converter.demosaic_batch(raws, p2, got, stream=st, graph=True)
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))


def test_host_io_batch_stream_and_graph_match_device_batch(converter):
    # pinned host buffers: per-slot copy streams; the graph records the
    # copies too, and its replays read the current contents of the same
    # host buffers
    st = torch.cuda.Stream()
    raws, params = _batch(400)
    ref = _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    st.synchronize()
    hraw = [r.cpu().pin_memory() for r in raws]
    hout = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in ref]
    converter.demosaic_batch(hraw, params, hout, stream=st)
    assert all(torch.equal(a.cuda(), b) for a, b in zip(hout, ref))
    for o in hout:
        o.zero_()
    converter.demosaic_batch(hraw, params, hout, stream=st, graph=True)  # runs and records
    assert all(torch.equal(a.cuda(), b) for a, b in zip(hout, ref))
    new_raws, _ = _batch(500)
    for h, n in zip(hraw, new_raws):
        h.copy_(n.cpu())
    ref2 = _outs()
    converter.demosaic_batch(new_raws, params, ref2, stream=st)
    st.synchronize()
    converter.demosaic_batch(hraw, params, hout, stream=st, graph=True)  # replays
    assert all(torch.equal(a.cuda(), b) for a, b in zip(hout, ref2))
