"""The FFMA2 pair form of the FP16 block matcher (the default one) and
its tile autotuner: the variants (thread rows x pixels per thread 8x4,
16x2 for 32 x 32 pixel tiles, 4x4, 8x2 for 32 x 16) compute the same bits
(same per-pixel arithmetic, same pairing, same centring vector), so forcing
any of them through GLS_BM_TILE, or letting the autotuner choose, gives
identical frames. Each setting runs in its own process because the kernel
choice and the variant are read once per process."""
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

_SCRIPT = r"""
import json, sys
import numpy as np, torch
import glasscamerapublic_b200 as g
from glasscamerapublic_b200 import RawConverter, scene
sizes = [(640, 480), (336, 250), (1000, 744)]
c = RawConverter(0)
st = torch.cuda.Stream()
raws, params, outs = [], [], []
for k, (w, h) in enumerate(sizes):
    wl = scene.Workload(f"t{k}", w, h, levels=5, gain=1.2 + 0.4 * k, read=3.0 + k, iso=800 * (k + 1), seed=70 + k)
    raw, _ = scene.make_raw(wl)
    raws.append(torch.from_numpy(raw.view(np.int16)).cuda())
    params.append(scene.make_params(wl))
    outs.append(torch.empty((h, w, 4), dtype=torch.float16, device="cuda"))
for rep in range(2):  # the second call reuses the chosen heights
    c.demosaic_batch(raws, params, outs, stream=st)
    st.synchronize()
    res = [o.cpu().numpy().view(np.uint16) for o in outs]
    np.savez(sys.argv[1] + f"_{rep}.npz", *res)
json.dump(g.block_match_tiles(), open(sys.argv[1] + ".json", "w"))
c.close()
"""


def _run(tmp_path, tag, tile):
    env = dict(os.environ)
    env.pop("GLS_BM_TILE", None)
    env.pop("GLS_BM_KERNEL", None)
    if tile:
        env["GLS_BM_TILE"] = str(tile)
    base = str(tmp_path / tag)
    subprocess.run([sys.executable, "-c", _SCRIPT, base], cwd=ROOT, env=env, check=True, timeout=300)
    frames = []
    for rep in range(2):
        with np.load(base + f"_{rep}.npz") as z:
            frames.append([z[k] for k in sorted(z.files, key=lambda s: int(s.split("_")[1]))])
    return frames, json.load(open(base + ".json"))


def test_tile_variants_are_bit_identical(tmp_path):
    ref, _ = _run(tmp_path, "v84", 84)
    for code in (44, 82, 162):
        got, _ = _run(tmp_path, f"v{code}", code)
        for rep in range(2):
            for a, b in zip(ref[rep], got[rep]):
                assert np.array_equal(a, b), code
    fa, tiles = _run(tmp_path, "auto", None)
    for rep in range(2):
        for a, c in zip(ref[rep], fa[rep]):
            assert np.array_equal(a, c)
    # the autotuner timed every FP16 pyramid level size it met
    assert tiles and all(t[2] in (84, 44, 82, 162) for t in tiles)
    sizes = {(t[0], t[1]) for t in tiles}
    assert (640, 480) in sizes and (320, 240) in sizes
