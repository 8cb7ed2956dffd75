"""The persistent batch kernel (GLS_PERSISTENT): every pyramid level of
every frame of a batch in one launch, from a device work list whose tasks
wait on per-level counters. It runs the stream kernels' device code (the
default block matcher's tile), so a batch of uneven frames gives the same
bits as the stream-launched batch, also when recorded and replayed as a
graph. Failure detection: a task
whose input never arrives ends its bounded wait with GLS_ERR_TIMEOUT and
leaves the device usable (no fault, no hang)."""
import ctypes as C

import numpy as np
import pytest
import torch

import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import scene

pytestmark = pytest.mark.gpu

# uneven sizes and level counts, down to levels smaller than a tile or a PCA patch
SIZES = [(320, 240, 5), (256, 192, 4), (200, 150, 3), (384, 288, 5), (72, 40, 3)]


def _batch(seed, iso=800):
    raws, params = [], []
    for k, (w, h, levels) in enumerate(SIZES):
        wl = scene.Workload(f"p{k}", w, h, levels=levels, gain=1.0 + 0.3 * k, read=3.0 + k, iso=iso, seed=seed + k,
                            white=4095 if k % 2 == 0 else 16383, black=512 if k % 2 == 0 else 2048)
        raw, _ = scene.make_raw(wl)
        raws.append(torch.from_numpy(raw.view(np.int16)).cuda())
        params.append(scene.make_params(wl))
    return raws, params


def _outs():
    return [torch.empty((h, w, 4), dtype=torch.float16, device="cuda") for (w, h, _) in SIZES]


def test_persistent_batch_bit_identical_to_stream_batch(converter):
    st = torch.cuda.Stream()
    raws, params = _batch(500)
    ref, got = _outs(), _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    converter.demosaic_batch(raws, params, got, stream=st, persistent=True)
    st.synchronize()
    for a, b in zip(ref, got):
        assert torch.equal(a, b)
    # the work list is reused for the same batch, and the result repeats
    for o in got:
        o.zero_()
    converter.demosaic_batch(raws, params, got, stream=st, persistent=True)
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))


def test_persistent_batch_recorded_as_graph(converter):
    st = torch.cuda.Stream()
    raws, params = _batch(600)
    ref, got = _outs(), _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    converter.demosaic_batch(raws, params, got, stream=st, persistent=True, graph=True)  # runs and records
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))
    new_raws, _ = _batch(700)
    for r, n in zip(raws, new_raws):
        r.copy_(n)
    converter.demosaic_batch(raws, params, ref, stream=st)
    for o in got:
        o.zero_()
    converter.demosaic_batch(raws, params, got, stream=st, persistent=True, graph=True)  # replays
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))


def test_persistent_batch_rejects_what_it_does_not_run(converter):
    raws, params = _batch(800)
    with pytest.raises(g.GlsError) as e:
        converter.demosaic_batch(raws, params, _outs(), fp16=False, out_fp16=False, persistent=True)
    assert e.value.code == g.GLS_ERR_INVALID_ARG
    host_raws = [r.cpu().numpy() for r in raws]
    host_outs = [o.cpu().numpy() for o in _outs()]
    with pytest.raises(g.GlsError) as e:  # host buffers
        converter.demosaic_batch(host_raws, params, host_outs, persistent=True)
    assert e.value.code == g.GLS_ERR_UNSUPPORTED


def test_persistent_wait_times_out_and_device_stays_usable(converter):
    err = C.c_int32(0)
    rc = g.lib().gls_persistent_selftest(0, 20_000_000, C.byref(err))  # 20 ms limit
    assert rc == g.GLS_ERR_TIMEOUT
    assert err.value == 3  # 1 + the eigen-solve task type
    assert b"wait ran out" in g.lib().gls_last_error_message()
    # the context still runs work: a persistent batch afterwards is correct
    st = torch.cuda.Stream()
    raws, params = _batch(900)
    ref, got = _outs(), _outs()
    converter.demosaic_batch(raws, params, ref, stream=st)
    converter.demosaic_batch(raws, params, got, stream=st, persistent=True)
    st.synchronize()
    assert all(torch.equal(a, b) for a, b in zip(ref, got))
