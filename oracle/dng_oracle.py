"""TEST INFRASTRUCTURE ONLY. An independent restatement, in plain Python,
of what the library's DNG ingest (glasscamerapublic_b200/csrc/gls_dng.cpp)
implements, for the tests to check it against:

  * a lossless JPEG codec (ITU-T T.81 process 14: Huffman-coded differences
    of predictors 1-7, any number of interleaved components, SSSS = 16 for a
    difference of 32768, byte stuffing), written from the specification;
  * a TIFF/DNG writer with options the library's writer never produces (big-
    endian byte order, the raw image in a SubIFD behind a thumbnail IFD0,
    10/12/14-bit packed samples, other predictors and component counts), so
    the reader meets files it did not write itself;
  * unpackDNGMetadata (MetalPipeline/demosaic_utils.cpp:268-366) with
    cam_xyz_coeff (:78-101) in float32, without automatic white balance, as
    CameraCalibration::getDemosaicParameters calls it
    (CameraCalibration.cpp:34-35).

The reference reads DNGs through its un-vendored GlassImage library, which
is not in the reference tree, so the reader itself is anchored on the
specifications, not on reference code: parity unpinned for the file reader;
the metadata-to-parameters step follows the reference's source.

Small images only (the codec is pure Python).
"""
from __future__ import annotations

import struct

import numpy as np

# ---------------------------------------------------------------- lossless JPEG


def _predict(pred, ra, rb, rc):
    return {1: ra, 2: rb, 3: rc, 4: ra + rb - rc, 5: ra + ((rb - rc) >> 1), 6: rb + ((ra - rc) >> 1),
            7: (ra + rb) >> 1}[pred]


def _category(d):
    d = int(d)
    return 16 if d == 32768 else abs(d).bit_length()


def _huffman_lengths(freq):
    """Code lengths (<= 16) for symbols 0..16 from frequencies (JPEG Annex K.2)."""
    syms = [s for s in range(17) if freq[s] > 0]
    if len(syms) == 1:
        return {syms[0]: 1}
    f = {s: freq[s] for s in syms}
    f[17] = 1  # reserved point: no all-ones code
    size = {s: 0 for s in f}
    groups = {s: [s] for s in f}
    while len(groups) > 1:
        a, b = sorted(groups, key=lambda s: (f[s], s))[:2]
        for s in groups[a] + groups[b]:
            size[s] += 1
        f[a] += f[b]
        groups[a] = groups[a] + groups[b]
        del groups[b], f[b]
    count = [0] * 40
    for s, l in size.items():
        count[l] += 1
    for i in range(39, 16, -1):
        while count[i] > 0:
            j = i - 2
            while count[j] == 0:
                j -= 1
            count[i] -= 2
            count[i - 1] += 1
            count[j + 1] += 2
            count[j] -= 1
    i = 16
    while count[i] == 0:
        i -= 1
    count[i] -= 1
    order = sorted((s for s in size if s != 17), key=lambda s: (size[s], s))
    lengths, k = {}, 0
    for l in range(1, 17):
        for _ in range(count[l]):
            lengths[order[k]] = l
            k += 1
    return lengths


def lj92_encode(samples: np.ndarray, predictor: int = 1, nc: int = 2, precision: int = 16) -> bytes:
    """samples (h, w): rows of w samples, coded as w / nc pixels of nc
    interleaved components."""
    h, w = samples.shape
    assert w % nc == 0
    X = w // nc
    s = samples.astype(np.int64).tolist()
    diffs = []
    for y in range(h):
        for x in range(X):
            for c in range(nc):
                k = x * nc + c
                if y == 0:
                    pv = s[y][k - nc] if x else 1 << (precision - 1)
                elif x == 0:
                    pv = s[y - 1][k]
                else:
                    pv = _predict(predictor, s[y][k - nc], s[y - 1][k], s[y - 1][k - nc])
                d = (s[y][k] - pv) & 0xFFFF
                if d > 32768:
                    d -= 65536
                diffs.append(d)
    freq = [0] * 17
    for d in diffs:
        freq[_category(d)] += 1
    lengths = _huffman_lengths(freq)
    bits = [0] * 16
    for l in lengths.values():
        bits[l - 1] += 1
    vals = sorted(lengths, key=lambda s: (lengths[s], s))
    codes, code = {}, 0
    k = 0
    for l in range(1, 17):
        for _ in range(bits[l - 1]):
            codes[vals[k]] = (code, l)
            code += 1
            k += 1
        code <<= 1
    out = bytearray(b"\xff\xd8")

    def seg(m, body):
        out.extend(bytes([0xFF, m]) + struct.pack(">H", len(body) + 2) + bytes(body))

    seg(0xC4, [0x00] + bits + vals)
    seg(0xC3, [precision] + list(struct.pack(">HH", h, X)) + [nc] + sum(([c + 1, 0x11, 0] for c in range(nc)), []))
    seg(0xDA, [nc] + sum(([c + 1, 0x00] for c in range(nc)), []) + [predictor, 0, 0])
    acc, n = 0, 0
    data = bytearray()
    for d in diffs:
        sz = _category(d)
        c, l = codes[sz]
        acc, n = (acc << l) | c, n + l
        if 0 < sz < 16:
            acc, n = (acc << sz) | (d + (1 << sz) - 1 if d < 0 else d), n + sz
        while n >= 8:
            b = (acc >> (n - 8)) & 0xFF
            data.append(b)
            if b == 0xFF:
                data.append(0)
            n -= 8
    if n:
        b = ((acc << (8 - n)) | ((1 << (8 - n)) - 1)) & 0xFF
        data.append(b)
        if b == 0xFF:
            data.append(0)
    out.extend(data)
    out.extend(b"\xff\xd9")
    return bytes(out)


def lj92_decode(data: bytes) -> np.ndarray:
    """(Y, X * Nc) samples of a lossless JPEG stream."""
    assert data[:2] == b"\xff\xd8"
    i = 2
    tables, comps, ctab = {}, [], {}
    P = X = Y = Nc = 0
    pred = pt = 1
    while True:
        m = data[i + 1]
        ln = struct.unpack(">H", data[i + 2:i + 4])[0]
        body = data[i + 4:i + 2 + ln]
        if m == 0xC4:
            k = 0
            while k < len(body):
                th = body[k] & 3
                bits = list(body[k + 1:k + 17])
                nv = sum(bits)
                vals = list(body[k + 17:k + 17 + nv])
                codes, code, j = {}, 0, 0
                for l in range(1, 17):
                    for _ in range(bits[l - 1]):
                        codes[(l, code)] = vals[j]
                        code += 1
                        j += 1
                    code <<= 1
                tables[th] = codes
                k += 17 + nv
        elif m == 0xC3:
            P, Y, X, Nc = body[0], struct.unpack(">H", body[1:3])[0], struct.unpack(">H", body[3:5])[0], body[5]
            comps = [body[6 + 3 * c] for c in range(Nc)]
        elif m == 0xDA:
            ns = body[0]
            for c in range(ns):
                ctab[comps.index(body[1 + 2 * c])] = body[2 + 2 * c] >> 4
            pred, pt = body[1 + 2 * ns], body[3 + 2 * ns] & 15
            i += 2 + ln
            break
        i += 2 + ln
    # entropy-coded bits, unstuffed
    bitstr = []
    j = i
    while j < len(data):
        b = data[j]
        if b == 0xFF:
            if data[j + 1] == 0:
                j += 2
            else:
                break
        else:
            j += 1
        bitstr.append(b)
    pos = [0]

    def bit():
        byte = bitstr[pos[0] >> 3] if (pos[0] >> 3) < len(bitstr) else 0
        v = (byte >> (7 - (pos[0] & 7))) & 1
        pos[0] += 1
        return v

    def get(k):
        v = 0
        for _ in range(k):
            v = (v << 1) | bit()
        return v

    out = np.zeros((Y, X * Nc), np.int64)
    for y in range(Y):
        for x in range(X):
            for c in range(Nc):
                codes = tables[ctab[c]]
                code, l = 0, 0
                while True:
                    code, l = (code << 1) | bit(), l + 1
                    if (l, code) in codes:
                        s = codes[(l, code)]
                        break
                if s == 16:
                    d = 32768
                elif s:
                    d = get(s)
                    if d < (1 << (s - 1)):
                        d -= (1 << s) - 1
                else:
                    d = 0
                k = x * Nc + c
                if y == 0:
                    pv = out[y, k - Nc] if x else 1 << (P - pt - 1)
                elif x == 0:
                    pv = out[y - 1, k]
                else:
                    pv = _predict(pred, int(out[y, k - Nc]), int(out[y - 1, k]), int(out[y - 1, k - Nc]))
                out[y, k] = (pv + d) & 0xFFFF
    return (out << pt).astype(np.uint16)


# ---------------------------------------------------------------- TIFF / DNG writer

_TYPES = {"B": 1, "A": 2, "H": 3, "L": 4, "R": 5, "SR": 10}


def _entry(tag, typ, values, bo):
    if typ == "A":
        raw = values.encode() + b"\0"
        return tag, 2, len(raw), raw
    if typ == "B":
        return tag, 1, len(values), bytes(values)
    if typ in ("R", "SR"):
        raw = b"".join(struct.pack(bo + ("ii" if typ == "SR" else "II"), int(round(v * 10000)), 10000)
                       for v in values)
        return tag, _TYPES[typ], len(values), raw
    raw = b"".join(struct.pack(bo + typ, v) for v in values)
    return tag, _TYPES[typ], len(values), raw


def _ifd(entries, bo, base, next_off=0):
    """An IFD at file offset base: (bytes, offsets of the value blocks by tag)."""
    entries = sorted(entries, key=lambda e: e[0])
    n = len(entries)
    data_at = base + 2 + 12 * n + 4
    head = struct.pack(bo + "H", n)
    tail = b""
    for tag, typ, count, raw in entries:
        if len(raw) <= 4:
            head += struct.pack(bo + "HHI", tag, typ, count) + raw.ljust(4, b"\0")
        else:
            head += struct.pack(bo + "HHI", tag, typ, count) + struct.pack(bo + "I", data_at + len(tail))
            tail += raw + (b"\0" if len(raw) & 1 else b"")
    return head + struct.pack(bo + "I", next_off) + tail


def pack_bits(raw: np.ndarray, bps: int) -> bytes:
    """Rows of bps-bit samples, most significant bit first, each row padded
    to a byte."""
    out = bytearray()
    for row in raw:
        acc, n = 0, 0
        for v in row:
            acc, n = (acc << bps) | int(v), n + bps
            while n >= 8:
                out.append((acc >> (n - 8)) & 0xFF)
                n -= 8
        if n:
            out.append((acc << (8 - n)) & 0xFF)
            acc, n = 0, 0
    return bytes(out)


def write_dng(path, raw: np.ndarray, meta: dict, big_endian=False, compression=7, tile=0, predictor=1, nc=2,
              bps=16, sub_ifd=True):
    """A DNG whose raw image sits in a SubIFD behind a thumbnail IFD0 (or in
    IFD0 with sub_ifd=False); LJ92 tiles (tile > 0) or one strip."""
    bo = ">" if big_endian else "<"
    h, w = raw.shape
    tw, th = (tile, tile) if tile else (w, h)
    pieces = []
    for ty in range(0, h, th):
        for tx in range(0, w, tw):
            t = np.zeros((th, tw), np.uint16)
            blk = raw[ty:ty + th, tx:tx + tw]
            t[:blk.shape[0], :blk.shape[1]] = blk
            if compression == 7:
                pieces.append(lj92_encode(t, predictor, nc))
            elif bps == 16:
                pieces.append(t.astype(bo + "u2").tobytes() if tile else raw.astype(bo + "u2").tobytes())
            else:
                pieces.append(pack_bits(t if tile else raw, bps))
            if not tile:
                break
        if not tile:
            break
    body = bytearray(b"MM\0*" if big_endian else b"II*\0") + b"\0\0\0\0"
    offs = []
    for p in pieces:
        while len(body) & 3:
            body.append(0)
        offs.append(len(body))
        body.extend(p)
    while len(body) & 3:
        body.append(0)
    exif_at = len(body)
    exif = [_entry(34855, "H", [meta.get("iso", 100)], bo), _entry(33434, "R", [meta.get("exposure_time", 0.01)], bo)]
    if meta.get("lens_model"):
        exif.append(_entry(42036, "A", meta["lens_model"], bo))
    body.extend(_ifd(exif, bo, exif_at))
    raw_entries = [
        _entry(254, "L", [0], bo), _entry(256, "L", [w], bo), _entry(257, "L", [h], bo),
        _entry(258, "H", [bps], bo), _entry(259, "H", [compression], bo), _entry(262, "H", [32803], bo),
        _entry(277, "H", [1], bo), _entry(33421, "H", [2, 2], bo), _entry(33422, "B", meta["cfa"], bo),
        _entry(50714, "R", [meta.get("black", 0)], bo), _entry(50717, "L", [meta.get("white", 65535)], bo)]
    if tile:
        raw_entries += [_entry(322, "L", [tw], bo), _entry(323, "L", [th], bo), _entry(324, "L", offs, bo),
                        _entry(325, "L", [len(p) for p in pieces], bo)]
    else:
        raw_entries += [_entry(273, "L", offs, bo), _entry(278, "L", [h], bo),
                        _entry(279, "L", [len(p) for p in pieces], bo)]
    main = [_entry(271, "A", meta.get("make", "Apple"), bo), _entry(272, "A", meta.get("model", "iPhone 14 Pro"), bo),
            _entry(50706, "B", [1, 4, 0, 0], bo), _entry(34665, "L", [exif_at], bo),
            _entry(50730, "SR", [meta.get("baseline_exposure", 0.0)], bo)]
    if "cm1" in meta:
        main.append(_entry(50721, "SR", meta["cm1"], bo))
    if "cm2" in meta:
        main.append(_entry(50722, "SR", meta["cm2"], bo))
    if "neutral" in meta:
        main.append(_entry(50728, "R", meta["neutral"], bo))
    while len(body) & 3:
        body.append(0)
    if sub_ifd:
        raw_at = len(body)
        body.extend(_ifd(raw_entries, bo, raw_at))
        while len(body) & 3:
            body.append(0)
        thumb = [_entry(254, "L", [1], bo), _entry(256, "L", [4], bo), _entry(257, "L", [4], bo),
                 _entry(262, "H", [2], bo), _entry(330, "L", [raw_at], bo)]
        ifd0_at = len(body)
        body.extend(_ifd(thumb + main, bo, ifd0_at))
    else:
        ifd0_at = len(body)
        body.extend(_ifd(raw_entries + main, bo, ifd0_at))
    body[4:8] = struct.pack(bo + "I", ifd0_at)
    with open(path, "wb") as f:
        f.write(bytes(body))


# ---------------------------------------------------------------- metadata -> parameters


def unpack_dng_metadata(cm, neutral, black, white, baseline_exposure, cfa, xyz_rgb):
    """(bayer, exposure_multiplier, rgb_cam (3, 3), scale_mul (4,)) in float32
    as unpackDNGMetadata computes them (auto_white_balance off): cam_xyz the
    DNG's colour matrix; cam_rgb = cam_xyz xyz_rgb; pre_mul = 1 / (cam_rgb
    (1, 1, 1)); rgb_cam = inverse(diag(pre_mul) cam_rgb); AsShotNeutral, where
    present, replaces pre_mul by its reciprocal; scale_mul[c] = max(2^BE, 1)
    (pre_mul[c] / min pre_mul) 65535 / (white - black), G2 taking G's."""
    f32 = np.float32
    cam_xyz = np.asarray(cm, f32).reshape(3, 3)
    xr = np.asarray(xyz_rgb, f32).reshape(3, 3)
    cam_rgb = np.zeros((3, 3), f32)
    for i in range(3):
        for j in range(3):
            s = f32(0)
            for k in range(3):
                s = f32(s + f32(cam_xyz[i, k] * xr[k, j]))
            cam_rgb[i, j] = s
    cam_white = np.array([f32(f32(cam_rgb[i, 0] + cam_rgb[i, 1]) + cam_rgb[i, 2]) for i in range(3)], f32)
    pre_mul = (f32(1) / cam_white).astype(f32)
    m = (np.diag(f32(1) / cam_white).astype(np.float64) @ cam_rgb.astype(np.float64))
    rgb_cam = np.linalg.inv(m).astype(f32)
    if neutral is not None:
        pre_mul = (f32(1) / np.asarray(neutral, f32)).astype(f32)
    em = f32(2.0 ** float(baseline_exposure))
    mn = pre_mul.min()
    scale = np.array([f32(float(f32(max(em, f32(1)) * f32(pre_mul[c if c < 3 else 1] / mn))) * 65535.0
                          / float(f32(white - black))) for c in range(4)], f32)
    bayer = {(0, 1, 1, 2): 2, (2, 1, 1, 0): 3, (1, 0, 2, 1): 0}.get(tuple(cfa), 1)
    return bayer, float(min(em, f32(1))), rgb_cam, scale
