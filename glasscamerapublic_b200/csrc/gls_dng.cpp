// gls_dng.cpp — DNG ingest: a TIFF/DNG reader and writer for the CFA raw
// image, with a lossless JPEG (ITU-T T.81 process 14) codec, and the DNG
// metadata -> DemosaicParameters step (unpackDNGMetadata,
// demosaic_utils.cpp:268-366; CameraCalibration::getDemosaicParameters,
// CameraCalibration.cpp:25-58). The reference reads DNGs through the
// un-vendored GlassImage library; this is a reader of its own, written
// from the TIFF 6.0, DNG 1.4 and T.81 specifications.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/glscam.h"
#include "gls_host.h"

namespace gls {
namespace {

// ---------------------------------------------------------------- TIFF
enum : uint16_t {
    T_NEWSUBFILETYPE = 254, T_WIDTH = 256, T_HEIGHT = 257, T_BPS = 258, T_COMPRESSION = 259, T_PHOTOMETRIC = 262,
    T_MAKE = 271, T_MODEL = 272, T_STRIPOFFSETS = 273, T_SPP = 277, T_ROWSPERSTRIP = 278, T_STRIPBYTES = 279,
    T_PLANAR = 284, T_TILEWIDTH = 322, T_TILELENGTH = 323, T_TILEOFFSETS = 324, T_TILEBYTES = 325, T_SUBIFDS = 330,
    T_CFAREPEAT = 33421, T_CFAPATTERN = 33422, T_EXPOSURETIME = 33434, T_EXIFIFD = 34665, T_ISO = 34855,
    T_REI = 34866, T_LENSMODEL = 42036, T_DNGVERSION = 50706, T_UNIQUEMODEL = 50708, T_BLACKLEVEL = 50714,
    T_WHITELEVEL = 50717, T_COLORMATRIX1 = 50721, T_COLORMATRIX2 = 50722, T_ASSHOTNEUTRAL = 50728,
    T_BASELINEEXPOSURE = 50730, T_ILLUMINANT1 = 50778, T_ILLUMINANT2 = 50779, T_ACTIVEAREA = 50829
};
constexpr uint16_t PHOTOMETRIC_CFA = 32803;

struct Entry {
    uint16_t type = 0;
    uint32_t count = 0;
    size_t data = 0;  // file offset of the value bytes
};
using Ifd = std::map<uint16_t, Entry>;

int type_size(uint16_t t) {
    switch (t) {
        case 1: case 2: case 6: case 7: return 1;
        case 3: case 8: return 2;
        case 4: case 9: case 11: case 13: return 4;
        case 5: case 10: case 12: return 8;
        default: return 0;
    }
}

struct File {
    std::vector<uint8_t> d;
    bool le = true;
    bool ok(size_t off, size_t len) const { return off <= d.size() && len <= d.size() - off; }
    uint16_t u16(size_t o) const {
        return le ? uint16_t(d[o] | d[o + 1] << 8) : uint16_t(d[o] << 8 | d[o + 1]);
    }
    uint32_t u32(size_t o) const {
        return le ? uint32_t(d[o]) | uint32_t(d[o + 1]) << 8 | uint32_t(d[o + 2]) << 16 | uint32_t(d[o + 3]) << 24
                  : uint32_t(d[o]) << 24 | uint32_t(d[o + 1]) << 16 | uint32_t(d[o + 2]) << 8 | uint32_t(d[o + 3]);
    }
    // the i-th value of an entry as a double (numeric types)
    double num(const Entry& e, uint32_t i) const {
        const size_t o = e.data + size_t(i) * type_size(e.type);
        switch (e.type) {
            case 1: case 7: return d[o];
            case 6: return int8_t(d[o]);
            case 3: return u16(o);
            case 8: return int16_t(u16(o));
            case 4: case 13: return u32(o);
            case 9: return int32_t(u32(o));
            case 5: { const uint32_t a = u32(o), b = u32(o + 4); return b ? double(a) / double(b) : 0.0; }
            case 10: { const int32_t a = int32_t(u32(o)), b = int32_t(u32(o + 4)); return b ? double(a) / double(b) : 0.0; }
            case 11: { const uint32_t u = u32(o); float f; std::memcpy(&f, &u, 4); return f; }
            case 12: {
                uint64_t u = le ? uint64_t(u32(o)) | uint64_t(u32(o + 4)) << 32 : uint64_t(u32(o)) << 32 | u32(o + 4);
                double f;
                std::memcpy(&f, &u, 8);
                return f;
            }
            default: return 0.0;
        }
    }
    std::vector<double> nums(const Ifd& ifd, uint16_t tag) const {
        std::vector<double> v;
        auto it = ifd.find(tag);
        if (it == ifd.end()) return v;
        for (uint32_t i = 0; i < it->second.count; i++) v.push_back(num(it->second, i));
        return v;
    }
    std::string str(const Ifd& ifd, uint16_t tag) const {
        auto it = ifd.find(tag);
        if (it == ifd.end()) return {};
        std::string s(reinterpret_cast<const char*>(&d[it->second.data]), it->second.count);
        const size_t z = s.find('\0');
        return z == std::string::npos ? s : s.substr(0, z);
    }
    bool parse_ifd(size_t off, Ifd& ifd, size_t* next) const {
        if (!ok(off, 2)) return false;
        const uint16_t n = u16(off);
        if (!ok(off + 2, size_t(n) * 12 + 4)) return false;
        for (uint16_t i = 0; i < n; i++) {
            const size_t eo = off + 2 + size_t(i) * 12;
            Entry e;
            e.type = u16(eo + 2);
            e.count = u32(eo + 4);
            const int ts = type_size(e.type);
            if (!ts) continue;
            const uint64_t bytes = uint64_t(ts) * e.count;
            e.data = bytes <= 4 ? eo + 8 : u32(eo + 8);
            if (!ok(e.data, size_t(bytes))) continue;
            ifd[u16(eo)] = e;
        }
        if (next) *next = u32(off + 2 + size_t(n) * 12);
        return true;
    }
};

// every IFD: the IFD0 chain, SubIFDs (recursively) and EXIF IFDs
void collect(const File& f, size_t off, int depth, std::vector<Ifd>& out, std::vector<Ifd>& exif) {
    for (int k = 0; off && k < 64 && depth < 4; k++) {
        Ifd ifd;
        size_t next = 0;
        if (!f.parse_ifd(off, ifd, &next)) return;
        out.push_back(ifd);
        for (double s : f.nums(ifd, T_SUBIFDS)) collect(f, size_t(s), depth + 1, out, exif);
        for (double e : f.nums(ifd, T_EXIFIFD)) {
            Ifd x;
            if (f.parse_ifd(size_t(e), x, nullptr)) exif.push_back(x);
        }
        off = next;
    }
}

// ---------------------------------------------------------------- lossless JPEG
struct Huff {
    // canonical code (T.81 Annex C): lookup of codes up to 9 bits, and per
    // length the largest code and the first value index
    uint16_t lut[512];  // (length << 8) | value, 0 = longer code
    int maxcode[18], valptr[17], mincode[17];
    uint8_t vals[256];
    bool ok = false;
    bool build(const uint8_t* bits, const uint8_t* hv, int nv) {
        std::memcpy(vals, hv, size_t(nv));
        std::fill(lut, lut + 512, uint16_t(0));
        int code = 0, k = 0;
        for (int l = 1; l <= 16; l++) {
            valptr[l] = k;
            mincode[l] = code;
            for (int i = 0; i < bits[l - 1]; i++, k++, code++) {
                if (code >= (1 << l) || k >= nv) return false;  // over-subscribed, or more codes than values
                if (l <= 9)
                    for (int f = 0; f < (1 << (9 - l)); f++) lut[(code << (9 - l)) | f] = uint16_t(l << 8 | vals[k]);
            }
            maxcode[l] = bits[l - 1] ? code - 1 : -1;
            code <<= 1;
        }
        maxcode[17] = 0x7fffffff;
        ok = k == nv;
        return ok;
    }
};

struct Bits {
    const uint8_t* p;
    size_t n, i = 0;
    uint64_t buf = 0;
    int cnt = 0;
    bool marker = false;  // a marker was met: feed zeros
    void fill() {
        while (cnt <= 56) {
            uint8_t b = 0;
            if (!marker && i < n) {
                b = p[i];
                if (b == 0xFF) {
                    const uint8_t nx = i + 1 < n ? p[i + 1] : 0;
                    if (nx == 0x00) {
                        i += 2;
                    } else {
                        marker = true;
                        b = 0;
                    }
                } else {
                    i++;
                }
            }
            buf |= uint64_t(b) << (56 - cnt);
            cnt += 8;
        }
    }
    int peek(int k) {
        if (cnt < k) fill();
        return int(buf >> (64 - k));
    }
    void skip(int k) {
        buf <<= k;
        cnt -= k;
    }
    int get(int k) {
        if (!k) return 0;
        const int v = peek(k);
        skip(k);
        return v;
    }
    int decode(const Huff& h) {
        const int l9 = peek(9);
        const uint16_t e = h.lut[l9];
        if (e) {
            skip(e >> 8);
            return e & 0xFF;
        }
        int code = get(1), l = 1;
        while (l < 16 && (h.maxcode[l] < 0 || code > h.maxcode[l])) {
            code = (code << 1) | get(1);
            l++;
        }
        if (h.maxcode[l] < 0 || code > h.maxcode[l]) return -1;
        return h.vals[h.valptr[l] + code - h.mincode[l]];
    }
};

// decodes one lossless JPEG stream: samples in scan order (Y rows of X
// pixels of Nc interleaved components)
bool lj92_decode(const uint8_t* p, size_t n, std::vector<uint16_t>& out, int* X_, int* Y_, int* Nc_, std::string& err) {
    if (n < 4 || p[0] != 0xFF || p[1] != 0xD8) return err = "no JPEG start marker", false;
    Huff tables[4];
    int P = 0, X = 0, Y = 0, Nc = 0, cid[4] = {}, ctab[4] = {}, pred = 1, pt = 0;
    size_t i = 2;
    bool scan = false;
    while (i + 4 <= n) {
        if (p[i] != 0xFF) return err = "bad JPEG marker", false;
        const uint8_t m = p[i + 1];
        const size_t len = size_t(p[i + 2]) << 8 | p[i + 3];
        if (i + 2 + len > n) return err = "truncated JPEG segment", false;
        const uint8_t* s = p + i + 4;
        if (m == 0xC4) {  // DHT
            size_t k = 0;
            while (k + 17 <= len - 2) {
                const int th = s[k] & 3;
                const uint8_t* bits = s + k + 1;
                int nv = 0;
                for (int l = 0; l < 16; l++) nv += bits[l];
                if (k + 17 + size_t(nv) > len - 2 || nv > 256) return err = "bad Huffman table", false;
                if (!tables[th].build(bits, s + k + 17, nv)) return err = "bad Huffman table", false;
                k += 17 + size_t(nv);
            }
        } else if (m == 0xC3) {  // SOF3
            P = s[0];
            Y = s[1] << 8 | s[2];
            X = s[3] << 8 | s[4];
            Nc = s[5];
            if (Nc < 1 || Nc > 4 || P < 2 || P > 16) return err = "unsupported lossless JPEG frame", false;
            for (int c = 0; c < Nc; c++) cid[c] = s[6 + 3 * c];
        } else if (m == 0xDA) {  // SOS
            const int ns = s[0];
            if (ns != Nc) return err = "scan components differ from the frame's", false;
            for (int c = 0; c < ns; c++) {
                const int id = s[1 + 2 * c], td = s[2 + 2 * c] >> 4;
                int idx = -1;
                for (int k = 0; k < Nc; k++)
                    if (cid[k] == id) idx = k;
                if (idx < 0 || td > 3) return err = "bad scan component", false;
                ctab[idx] = td;
            }
            pred = s[1 + 2 * ns];
            pt = s[3 + 2 * ns] & 15;
            i += 2 + len;
            scan = true;
            break;
        } else if (m == 0xDD) {
            return err = "restart intervals are not supported", false;
        } else if (m >= 0xC0 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC) {
            return err = "not a lossless (process 14) JPEG", false;
        }
        i += 2 + len;
    }
    if (!scan || !X || !Y) return err = "no JPEG scan", false;
    if (pred < 1 || pred > 7) return err = "bad lossless predictor", false;
    for (int c = 0; c < Nc; c++)
        if (!tables[ctab[c]].ok) return err = "missing Huffman table", false;
    const size_t row = size_t(X) * Nc;
    out.assign(row * size_t(Y), 0);
    Bits b{p + i, n - i};
    const int init = 1 << (P - pt - 1);
    for (int y = 0; y < Y; y++) {
        uint16_t* r = &out[size_t(y) * row];
        const uint16_t* up = y ? r - row : nullptr;
        for (int x = 0; x < X; x++)
            for (int c = 0; c < Nc; c++) {
                const int ssss = b.decode(tables[ctab[c]]);
                if (ssss < 0 || ssss > 16) return err = "bad Huffman code", false;
                int diff = 0;
                if (ssss == 16) {
                    diff = 32768;
                } else if (ssss) {
                    diff = b.get(ssss);
                    if (diff < (1 << (ssss - 1))) diff -= (1 << ssss) - 1;
                }
                const size_t k = size_t(x) * Nc + c;
                int pv;
                if (!y) {
                    pv = x ? r[k - Nc] : init;
                } else if (!x) {
                    pv = up[k];
                } else {
                    const int ra = r[k - Nc], rb = up[k], rc = up[k - Nc];
                    switch (pred) {
                        case 1: pv = ra; break;
                        case 2: pv = rb; break;
                        case 3: pv = rc; break;
                        case 4: pv = ra + rb - rc; break;
                        case 5: pv = ra + ((rb - rc) >> 1); break;
                        case 6: pv = rb + ((ra - rc) >> 1); break;
                        default: pv = (ra + rb) >> 1; break;
                    }
                }
                r[k] = uint16_t((pv + diff) & 0xFFFF);
            }
    }
    if (pt)
        for (auto& v : out) v = uint16_t(v << pt);
    *X_ = X;
    *Y_ = Y;
    *Nc_ = Nc;
    return true;
}

// ---- encoder (predictor 1, 16-bit precision)
struct BitWriter {
    std::vector<uint8_t>& o;
    uint64_t buf = 0;
    int cnt = 0;
    void put(uint32_t v, int k) {
        if (!k) return;
        buf = (buf << k) | (v & ((1u << k) - 1));
        cnt += k;
        while (cnt >= 8) {
            const uint8_t b = uint8_t(buf >> (cnt - 8));
            o.push_back(b);
            if (b == 0xFF) o.push_back(0);
            cnt -= 8;
        }
    }
    void flush() {
        if (cnt) put((1u << (8 - cnt)) - 1, 8 - cnt);  // pad with ones
    }
};

int category(int d) {
    if (d == 32768) return 16;
    int a = d < 0 ? -d : d, s = 0;
    while (a) {
        s++;
        a >>= 1;
    }
    return s;
}

// JPEG Annex K.2: code lengths from frequencies, limited to 16 bits
void code_lengths(const long freq_in[17], uint8_t bits[16], uint8_t vals[17], int* nv) {
    long freq[18];
    for (int i = 0; i < 17; i++) freq[i] = freq_in[i];
    freq[17] = 1;  // the reserved code point, so no code is all ones
    int codesize[18] = {}, others[18];
    for (int i = 0; i < 18; i++) others[i] = -1;
    for (;;) {
        int v1 = -1, v2 = -1;
        for (int i = 0; i < 18; i++)
            if (freq[i] > 0 && (v1 < 0 || freq[i] <= freq[v1])) v1 = i;
        for (int i = 0; i < 18; i++)
            if (i != v1 && freq[i] > 0 && (v2 < 0 || freq[i] <= freq[v2])) v2 = i;
        if (v2 < 0) break;
        freq[v1] += freq[v2];
        freq[v2] = 0;
        codesize[v1]++;
        while (others[v1] >= 0) {
            v1 = others[v1];
            codesize[v1]++;
        }
        others[v1] = v2;
        codesize[v2]++;
        while (others[v2] >= 0) {
            v2 = others[v2];
            codesize[v2]++;
        }
    }
    int count[33] = {};
    for (int i = 0; i < 18; i++)
        if (codesize[i]) count[codesize[i]]++;
    for (int i = 32; i > 16; i--)
        while (count[i] > 0) {
            int j = i - 2;
            while (count[j] == 0) j--;
            count[i] -= 2;
            count[i - 1]++;
            count[j + 1] += 2;
            count[j]--;
        }
    int i = 16;
    while (count[i] == 0) i--;
    count[i]--;  // drop the reserved code point
    for (int l = 0; l < 16; l++) bits[l] = uint8_t(count[l + 1]);
    int k = 0;
    for (int l = 1; l <= 32; l++)
        for (int s = 0; s < 17; s++)
            if (codesize[s] == l) vals[k++] = uint8_t(s);
    *nv = k;
}

// one tile (w x h samples, w even) as a lossless JPEG of w/2 two-component
// pixels per row
std::vector<uint8_t> lj92_encode(const uint16_t* src, size_t stride, int w, int h) {
    const int Nc = (w % 2 == 0) ? 2 : 1, X = w / Nc;
    std::vector<int> diffs(size_t(w) * h);
    long freq[17] = {};
    for (int y = 0; y < h; y++)
        for (int x = 0; x < X; x++)
            for (int c = 0; c < Nc; c++) {
                const int k = x * Nc + c;
                const int v = src[size_t(y) * stride + k];
                const int pv = !y ? (x ? src[size_t(y) * stride + k - Nc] : 1 << 15)
                                  : (!x ? src[size_t(y - 1) * stride + k] : src[size_t(y) * stride + k - Nc]);
                int d = (v - pv) & 0xFFFF;
                if (d > 32768) d -= 65536;
                diffs[size_t(y) * w + k] = d;
                freq[category(d)]++;
            }
    uint8_t bits[16], vals[17];
    int nv = 0;
    code_lengths(freq, bits, vals, &nv);
    int code_of[17] = {}, len_of[17] = {};
    {
        int code = 0, k = 0;
        for (int l = 1; l <= 16; l++) {
            for (int i = 0; i < bits[l - 1]; i++, k++) {
                code_of[vals[k]] = code++;
                len_of[vals[k]] = l;
            }
            code <<= 1;
        }
    }
    std::vector<uint8_t> o = {0xFF, 0xD8};
    auto seg = [&](uint8_t m, const std::vector<uint8_t>& body) {
        o.push_back(0xFF);
        o.push_back(m);
        o.push_back(uint8_t((body.size() + 2) >> 8));
        o.push_back(uint8_t(body.size() + 2));
        o.insert(o.end(), body.begin(), body.end());
    };
    std::vector<uint8_t> dht = {0x00};
    dht.insert(dht.end(), bits, bits + 16);
    dht.insert(dht.end(), vals, vals + nv);
    seg(0xC4, dht);
    std::vector<uint8_t> sof = {16, uint8_t(h >> 8), uint8_t(h), uint8_t(X >> 8), uint8_t(X), uint8_t(Nc)};
    for (int c = 0; c < Nc; c++) sof.insert(sof.end(), {uint8_t(c), 0x11, 0});
    seg(0xC3, sof);
    std::vector<uint8_t> sos = {uint8_t(Nc)};
    for (int c = 0; c < Nc; c++) sos.insert(sos.end(), {uint8_t(c), 0x00});
    sos.insert(sos.end(), {1, 0, 0});  // predictor 1, point transform 0
    seg(0xDA, sos);
    BitWriter bw{o};
    for (int d : diffs) {
        const int s = category(d);
        bw.put(uint32_t(code_of[s]), len_of[s]);
        if (s && s < 16) bw.put(uint32_t(d < 0 ? d + (1 << s) - 1 : d), s);
    }
    bw.flush();
    o.push_back(0xFF);
    o.push_back(0xD9);
    return o;
}

// ---------------------------------------------------------------- helpers
bool read_file(const char* path, std::vector<uint8_t>& d) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    d.resize(n > 0 ? size_t(n) : 0);
    const size_t got = d.empty() ? 0 : std::fread(d.data(), 1, d.size(), f);
    std::fclose(f);
    return got == d.size();
}

// the Bayer pattern as unpackDNGMetadata maps CFAPattern
// (demosaic_utils.cpp:295-298): anything but RGGB, BGGR and GRBG is GBRG
int bayer_of(const uint8_t* cfa) {
    static const uint8_t rggb[4] = {0, 1, 1, 2}, bggr[4] = {2, 1, 1, 0}, grbg[4] = {1, 0, 2, 1};
    if (!std::memcmp(cfa, rggb, 4)) return GLS_RGGB;
    if (!std::memcmp(cfa, bggr, 4)) return GLS_BGGR;
    if (!std::memcmp(cfa, grbg, 4)) return GLS_GRBG;
    return GLS_GBRG;
}

}  // namespace
}  // namespace gls

using namespace gls;

extern "C" gls_status gls_dng_read(const char* path, gls_dng_info* info, uint16_t* raw, size_t raw_stride_elems) {
    clear_error();
    if (!path || !info) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    File f;
    if (!read_file(path, f.d)) return set_error(GLS_ERR_INVALID_ARG, "cannot read %s", path);
    if (f.d.size() < 8) return set_error(GLS_ERR_INVALID_ARG, "%s: not a TIFF file", path);
    if (f.d[0] == 'I' && f.d[1] == 'I') f.le = true;
    else if (f.d[0] == 'M' && f.d[1] == 'M') f.le = false;
    else return set_error(GLS_ERR_INVALID_ARG, "%s: not a TIFF file", path);
    if (f.u16(2) != 42) return set_error(GLS_ERR_INVALID_ARG, "%s: not a TIFF file", path);
    std::vector<Ifd> ifds, exifs;
    collect(f, f.u32(4), 0, ifds, exifs);
    if (ifds.empty()) return set_error(GLS_ERR_INVALID_ARG, "%s: no IFD", path);
    const Ifd* rawifd = nullptr;
    for (const Ifd& d : ifds) {
        const auto st = f.nums(d, T_NEWSUBFILETYPE), ph = f.nums(d, T_PHOTOMETRIC);
        if ((st.empty() || st[0] == 0) && !ph.empty() && ph[0] == PHOTOMETRIC_CFA) {
            rawifd = &d;
            break;
        }
    }
    if (!rawifd) return set_error(GLS_ERR_UNSUPPORTED, "%s: no CFA raw image", path);
    const Ifd& ri = *rawifd;
    const Ifd& i0 = ifds[0];
    auto first = [&](const Ifd& d, uint16_t tag, double def) {
        const auto v = f.nums(d, tag);
        return v.empty() ? def : v[0];
    };
    auto any = [&](uint16_t tag) -> const Ifd* {  // the raw IFD first, then IFD0
        if (ri.count(tag)) return &ri;
        if (i0.count(tag)) return &i0;
        return nullptr;
    };
    gls_dng_info in{};
    in.width = int32_t(first(ri, T_WIDTH, 0));
    in.height = int32_t(first(ri, T_HEIGHT, 0));
    in.bits_per_sample = int32_t(first(ri, T_BPS, 16));
    in.compression = int32_t(first(ri, T_COMPRESSION, 1));
    if (in.width <= 0 || in.height <= 0) return set_error(GLS_ERR_INVALID_ARG, "%s: bad raw size", path);
    if (first(ri, T_SPP, 1) != 1) return set_error(GLS_ERR_UNSUPPORTED, "%s: more than one sample per pixel", path);
    {
        const auto rep = f.nums(ri, T_CFAREPEAT);
        const auto cfa = f.nums(ri, T_CFAPATTERN);
        if ((!rep.empty() && (rep.size() < 2 || rep[0] != 2 || rep[1] != 2)) || cfa.size() < 4)
            return set_error(GLS_ERR_UNSUPPORTED, "%s: not a 2x2 Bayer CFA", path);
        for (int c = 0; c < 4; c++) in.cfa_pattern[c] = uint8_t(cfa[c]);
        in.bayer_pattern = bayer_of(in.cfa_pattern);
    }
    const Ifd* d;
    in.black_level = (d = any(T_BLACKLEVEL)) ? float(first(*d, T_BLACKLEVEL, 0)) : 0.f;
    in.white_level = (d = any(T_WHITELEVEL)) ? float(first(*d, T_WHITELEVEL, 65535)) : 65535.f;
    in.baseline_exposure = float(first(i0, T_BASELINEEXPOSURE, 0));
    for (int k = 0; k < 2; k++) {
        const auto m = f.nums(i0, k ? T_COLORMATRIX2 : T_COLORMATRIX1);
        if (m.size() >= 9) {
            (k ? in.has_color_matrix2 : in.has_color_matrix1) = 1;
            for (int j = 0; j < 9; j++) (k ? in.color_matrix2 : in.color_matrix1)[j] = float(m[j]);
        }
    }
    {
        const auto n = f.nums(i0, T_ASSHOTNEUTRAL);
        if (n.size() >= 3) {
            in.has_as_shot_neutral = 1;
            for (int c = 0; c < 3; c++) in.as_shot_neutral[c] = float(n[c]);
        }
    }
    in.calibration_illuminant1 = int32_t(first(i0, T_ILLUMINANT1, 0));
    in.calibration_illuminant2 = int32_t(first(i0, T_ILLUMINANT2, 0));
    // ISO as CameraCalibration::getDemosaicParameters takes it (:38-46)
    for (const Ifd& x : exifs) {
        if (!in.iso && x.count(T_REI)) in.iso = int32_t(first(x, T_REI, 0));
        if (!in.iso && x.count(T_ISO)) in.iso = int32_t(first(x, T_ISO, 0));
        if (in.exposure_time == 0.f) in.exposure_time = float(first(x, T_EXPOSURETIME, 0));
        if (!in.lens_model[0]) std::snprintf(in.lens_model, sizeof(in.lens_model), "%s", f.str(x, T_LENSMODEL).c_str());
    }
    if (!in.iso) in.iso = int32_t(first(i0, T_ISO, 0));
    {
        const auto a = f.nums(ri, T_ACTIVEAREA);
        if (a.size() >= 4) for (int k = 0; k < 4; k++) in.active_area[k] = int32_t(a[k]);
        else in.active_area[0] = 0, in.active_area[1] = 0, in.active_area[2] = in.height, in.active_area[3] = in.width;
    }
    std::snprintf(in.make, sizeof(in.make), "%s", f.str(i0, T_MAKE).c_str());
    std::snprintf(in.model, sizeof(in.model), "%s", f.str(i0, T_MODEL).c_str());
    *info = in;
    if (!raw) return GLS_OK;
    if (raw_stride_elems < size_t(in.width)) return set_error(GLS_ERR_INVALID_ARG, "raw stride too small");

    // the pieces: tiles, or strips (full-width tiles)
    const bool tiled = ri.count(T_TILEOFFSETS) != 0;
    const int tw = tiled ? int(first(ri, T_TILEWIDTH, 0)) : in.width;
    const int th = tiled ? int(first(ri, T_TILELENGTH, 0)) : int(first(ri, T_ROWSPERSTRIP, in.height));
    const auto offs = f.nums(ri, tiled ? T_TILEOFFSETS : T_STRIPOFFSETS);
    const auto cnts = f.nums(ri, tiled ? T_TILEBYTES : T_STRIPBYTES);
    if (tw <= 0 || th <= 0 || offs.empty() || offs.size() != cnts.size())
        return set_error(GLS_ERR_INVALID_ARG, "%s: bad raw layout", path);
    const int tx_n = (in.width + tw - 1) / tw, ty_n = (in.height + th - 1) / th;
    if (offs.size() < size_t(tx_n) * ty_n) return set_error(GLS_ERR_INVALID_ARG, "%s: missing raw pieces", path);
    const int bps = in.bits_per_sample, comp = in.compression;
    if (comp != 1 && comp != 7) return set_error(GLS_ERR_UNSUPPORTED, "%s: compression %d", path, comp);
    if (comp == 1 && (bps < 8 || bps > 16)) return set_error(GLS_ERR_UNSUPPORTED, "%s: %d bits per sample", path, bps);
    std::atomic<int> next{0}, failed{0};
    std::string first_err;
    std::atomic<bool> err_set{false};
    auto work = [&]() {
        std::vector<uint16_t> buf;
        std::string err;
        for (int t; (t = next.fetch_add(1)) < tx_n * ty_n && !failed.load();) {
            const int x0 = (t % tx_n) * tw, y0 = (t / tx_n) * th;
            const int pw = std::min(tw, in.width - x0), ph = std::min(th, in.height - y0);
            const size_t off = size_t(offs[t]), len = size_t(cnts[t]);
            if (!f.ok(off, len)) {
                err = "raw piece outside the file";
            } else if (comp == 7) {
                int X = 0, Y = 0, Nc = 0;
                if (lj92_decode(&f.d[off], len, buf, &X, &Y, &Nc, err)) {
                    // the decoded samples fill the tile row by row (a tile's
                    // JPEG may interleave two rows or two components)
                    const size_t total = buf.size();
                    for (size_t i = 0; i < total; i++) {
                        const int yy = int(i / size_t(tw)), xx = int(i % size_t(tw));
                        if (yy >= ph) break;
                        if (xx < pw) raw[size_t(y0 + yy) * raw_stride_elems + x0 + xx] = buf[i];
                    }
                    continue;
                }
            } else {
                const size_t row_bytes = (size_t(tw) * bps + 7) / 8;
                if (len < row_bytes * size_t(ph) - (row_bytes - (size_t(pw) * bps + 7) / 8)) {
                    err = "raw piece too short";
                } else {
                    const uint8_t* src = &f.d[off];
                    for (int yy = 0; yy < ph; yy++) {
                        const uint8_t* r = src + size_t(yy) * row_bytes;
                        uint16_t* o = raw + size_t(y0 + yy) * raw_stride_elems + x0;
                        if (bps == 16) {
                            for (int xx = 0; xx < pw; xx++)
                                o[xx] = f.le ? uint16_t(r[2 * xx] | r[2 * xx + 1] << 8) : uint16_t(r[2 * xx] << 8 | r[2 * xx + 1]);
                        } else if (bps == 8) {
                            for (int xx = 0; xx < pw; xx++) o[xx] = r[xx];
                        } else {  // packed, most significant bit first
                            size_t bit = 0;
                            for (int xx = 0; xx < pw; xx++) {
                                uint32_t v = 0;
                                for (int k = 0; k < bps; k++, bit++) v = (v << 1) | ((r[bit >> 3] >> (7 - (bit & 7))) & 1);
                                o[xx] = uint16_t(v);
                            }
                        }
                    }
                    continue;
                }
            }
            failed = 1;
            if (!err_set.exchange(true)) first_err = err;
        }
    };
    const int nt = std::max(1, std::min<int>(int(std::thread::hardware_concurrency()), tx_n * ty_n));
    std::vector<std::thread> pool;
    for (int k = 1; k < nt; k++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
    if (failed) return set_error(GLS_ERR_INVALID_ARG, "%s: %s", path, first_err.c_str());
    return GLS_OK;
}

namespace {
struct TiffOut {
    std::vector<uint8_t> d;
    void u16(uint16_t v) { d.push_back(uint8_t(v)), d.push_back(uint8_t(v >> 8)); }
    void u32(uint32_t v) { for (int k = 0; k < 4; k++) d.push_back(uint8_t(v >> (8 * k))); }
    void at32(size_t o, uint32_t v) { for (int k = 0; k < 4; k++) d[o + k] = uint8_t(v >> (8 * k)); }
    void pad() { while (d.size() & 3) d.push_back(0); }
};
struct OutEntry {
    uint16_t tag, type;
    uint32_t count;
    std::vector<uint8_t> bytes;  // little-endian value bytes
};
OutEntry e_short(uint16_t tag, std::vector<uint32_t> v) {
    OutEntry e{tag, 3, uint32_t(v.size()), {}};
    for (uint32_t x : v) e.bytes.push_back(uint8_t(x)), e.bytes.push_back(uint8_t(x >> 8));
    return e;
}
OutEntry e_long(uint16_t tag, std::vector<uint32_t> v) {
    OutEntry e{tag, 4, uint32_t(v.size()), {}};
    for (uint32_t x : v) for (int k = 0; k < 4; k++) e.bytes.push_back(uint8_t(x >> (8 * k)));
    return e;
}
OutEntry e_bytes(uint16_t tag, uint16_t type, std::vector<uint8_t> v) { return {tag, type, uint32_t(v.size()), v}; }
OutEntry e_ascii(uint16_t tag, const char* s) {
    std::vector<uint8_t> v(s, s + std::strlen(s));
    v.push_back(0);
    return {tag, 2, uint32_t(v.size()), v};
}
OutEntry e_srational(uint16_t tag, const float* v, int n, bool sign = true) {
    OutEntry e{tag, uint16_t(sign ? 10 : 5), uint32_t(n), {}};
    for (int i = 0; i < n; i++) {
        const int32_t num = int32_t(std::lround(double(v[i]) * 1000000.0)), den = 1000000;
        for (int k = 0; k < 4; k++) e.bytes.push_back(uint8_t(uint32_t(num) >> (8 * k)));
        for (int k = 0; k < 4; k++) e.bytes.push_back(uint8_t(uint32_t(den) >> (8 * k)));
    }
    return e;
}
// writes an IFD (entries sorted by tag) at the end of t; returns its offset.
// Value blocks longer than 4 bytes go after the IFD.
size_t write_ifd(TiffOut& t, std::vector<OutEntry> es, uint32_t next) {
    std::sort(es.begin(), es.end(), [](const OutEntry& a, const OutEntry& b) { return a.tag < b.tag; });
    t.pad();
    const size_t at = t.d.size();
    const size_t data0 = at + 2 + es.size() * 12 + 4;
    size_t data = data0;
    std::vector<size_t> where(es.size());
    for (size_t i = 0; i < es.size(); i++)
        if (es[i].bytes.size() > 4) {
            where[i] = data;
            data += (es[i].bytes.size() + 1) & ~size_t(1);
        }
    t.u16(uint16_t(es.size()));
    for (size_t i = 0; i < es.size(); i++) {
        t.u16(es[i].tag);
        t.u16(es[i].type);
        t.u32(es[i].count);
        if (es[i].bytes.size() > 4) {
            t.u32(uint32_t(where[i]));
        } else {
            std::vector<uint8_t> b = es[i].bytes;
            b.resize(4, 0);
            t.d.insert(t.d.end(), b.begin(), b.end());
        }
    }
    t.u32(next);
    for (size_t i = 0; i < es.size(); i++)
        if (es[i].bytes.size() > 4) {
            t.d.insert(t.d.end(), es[i].bytes.begin(), es[i].bytes.end());
            if (es[i].bytes.size() & 1) t.d.push_back(0);
        }
    return at;
}
}  // namespace

extern "C" gls_status gls_dng_write(const char* path, const gls_dng_info* info, const uint16_t* raw,
                                    size_t raw_stride_elems, int32_t compression, int32_t tile_size) {
    clear_error();
    if (!path || !info || !raw) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    const int W = info->width, H = info->height;
    if (W <= 0 || H <= 0 || raw_stride_elems < size_t(W)) return set_error(GLS_ERR_INVALID_ARG, "bad raw size");
    if (compression != 1 && compression != 7) return set_error(GLS_ERR_UNSUPPORTED, "compression %d", compression);
    if (tile_size < 0 || (tile_size && (tile_size % 16))) return set_error(GLS_ERR_INVALID_ARG, "tile size must be a multiple of 16");
    const bool tiled = tile_size > 0;
    const int tw = tiled ? tile_size : W, th = tiled ? tile_size : H;
    const int tx_n = (W + tw - 1) / tw, ty_n = (H + th - 1) / th;
    // the pieces' bytes
    std::vector<std::vector<uint8_t>> pieces(size_t(tx_n) * ty_n);
    auto encode = [&](int t) {
        const int x0 = (t % tx_n) * tw, y0 = (t / tx_n) * th;
        std::vector<uint16_t> tile(size_t(tw) * th, 0);  // edge tiles padded by repeating the last sample
        for (int y = 0; y < th; y++)
            for (int x = 0; x < tw; x++)
                tile[size_t(y) * tw + x] = raw[size_t(std::min(y0 + y, H - 1)) * raw_stride_elems + std::min(x0 + x, W - 1)];
        if (compression == 7) {
            pieces[t] = lj92_encode(tile.data(), size_t(tw), tw, th);
        } else {
            auto& p = pieces[t];
            const int ph = tiled ? th : H;
            p.resize(size_t(tw) * ph * 2);
            for (size_t i = 0; i < size_t(tw) * ph; i++) p[2 * i] = uint8_t(tile[i]), p[2 * i + 1] = uint8_t(tile[i] >> 8);
        }
    };
    {
        std::atomic<int> next{0};
        auto work = [&]() {
            for (int t; (t = next.fetch_add(1)) < tx_n * ty_n;) encode(t);
        };
        const int nt = std::max(1, std::min<int>(int(std::thread::hardware_concurrency()), tx_n * ty_n));
        std::vector<std::thread> pool;
        for (int k = 1; k < nt; k++) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
    }
    TiffOut t;
    t.d = {'I', 'I', 42, 0, 0, 0, 0, 0};
    std::vector<uint32_t> offs, cnts;
    for (auto& p : pieces) {
        t.pad();
        offs.push_back(uint32_t(t.d.size()));
        cnts.push_back(uint32_t(p.size()));
        t.d.insert(t.d.end(), p.begin(), p.end());
    }
    // EXIF IFD
    std::vector<OutEntry> ex;
    if (info->iso > 0) {
        ex.push_back(e_short(T_ISO, {uint32_t(std::min(info->iso, 65535))}));
        ex.push_back(e_long(T_REI, {uint32_t(info->iso)}));
    }
    if (info->exposure_time > 0) ex.push_back(e_srational(T_EXPOSURETIME, &info->exposure_time, 1, false));
    if (info->lens_model[0]) ex.push_back(e_ascii(T_LENSMODEL, info->lens_model));
    if (ex.empty()) ex.push_back(e_short(T_ISO, {0}));
    const size_t exif_at = write_ifd(t, ex, 0);
    std::vector<OutEntry> es;
    es.push_back(e_long(T_NEWSUBFILETYPE, {0}));
    es.push_back(e_long(T_WIDTH, {uint32_t(W)}));
    es.push_back(e_long(T_HEIGHT, {uint32_t(H)}));
    es.push_back(e_short(T_BPS, {16}));
    es.push_back(e_short(T_COMPRESSION, {uint32_t(compression)}));
    es.push_back(e_short(T_PHOTOMETRIC, {PHOTOMETRIC_CFA}));
    if (info->make[0]) es.push_back(e_ascii(T_MAKE, info->make));
    if (info->model[0]) es.push_back(e_ascii(T_MODEL, info->model));
    es.push_back(e_short(T_SPP, {1}));
    es.push_back(e_short(T_PLANAR, {1}));
    if (tiled) {
        es.push_back(e_long(T_TILEWIDTH, {uint32_t(tw)}));
        es.push_back(e_long(T_TILELENGTH, {uint32_t(th)}));
        es.push_back(e_long(T_TILEOFFSETS, offs));
        es.push_back(e_long(T_TILEBYTES, cnts));
    } else {
        es.push_back(e_long(T_STRIPOFFSETS, offs));
        es.push_back(e_long(T_ROWSPERSTRIP, {uint32_t(H)}));
        es.push_back(e_long(T_STRIPBYTES, cnts));
    }
    es.push_back(e_short(T_CFAREPEAT, {2, 2}));
    es.push_back(e_bytes(T_CFAPATTERN, 1, {info->cfa_pattern[0], info->cfa_pattern[1], info->cfa_pattern[2],
                                           info->cfa_pattern[3]}));
    es.push_back(e_long(T_EXIFIFD, {uint32_t(exif_at)}));
    es.push_back(e_bytes(T_DNGVERSION, 1, {1, 4, 0, 0}));
    es.push_back(e_ascii(T_UNIQUEMODEL, info->model[0] ? info->model : "B200 raw"));
    es.push_back(e_srational(T_BLACKLEVEL, &info->black_level, 1, false));
    es.push_back(e_long(T_WHITELEVEL, {uint32_t(info->white_level)}));
    if (info->has_color_matrix1) es.push_back(e_srational(T_COLORMATRIX1, info->color_matrix1, 9));
    if (info->has_color_matrix2) es.push_back(e_srational(T_COLORMATRIX2, info->color_matrix2, 9));
    if (info->has_as_shot_neutral) es.push_back(e_srational(T_ASSHOTNEUTRAL, info->as_shot_neutral, 3, false));
    es.push_back(e_srational(T_BASELINEEXPOSURE, &info->baseline_exposure, 1));
    if (info->calibration_illuminant1) es.push_back(e_short(T_ILLUMINANT1, {uint32_t(info->calibration_illuminant1)}));
    if (info->calibration_illuminant2) es.push_back(e_short(T_ILLUMINANT2, {uint32_t(info->calibration_illuminant2)}));
    const size_t ifd0 = write_ifd(t, es, 0);
    t.at32(4, uint32_t(ifd0));
    FILE* fo = std::fopen(path, "wb");
    if (!fo) return set_error(GLS_ERR_INVALID_ARG, "cannot write %s", path);
    const size_t put = std::fwrite(t.d.data(), 1, t.d.size(), fo);
    std::fclose(fo);
    if (put != t.d.size()) return set_error(GLS_ERR_INVALID_ARG, "short write to %s", path);
    return GLS_OK;
}

// ---------------------------------------------------------------- metadata -> parameters
namespace {
using M3 = std::array<std::array<float, 3>, 3>;
M3 mul3(const M3& a, const M3& b) {
    M3 r{};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            float s = 0;
            for (int k = 0; k < 3; k++) s += a[i][k] * b[k][j];
            r[i][j] = s;
        }
    return r;
}
bool inv3(const M3& m, M3& r) {
    const float a = m[0][0], b = m[0][1], c = m[0][2], d = m[1][0], e = m[1][1], f = m[1][2], g = m[2][0],
                h = m[2][1], i = m[2][2];
    const float A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
    const float det = a * A + b * B + c * C;
    if (det == 0.f) return false;
    r = {{{A / det, -(b * i - c * h) / det, (b * f - c * e) / det},
          {B / det, (a * i - c * g) / det, -(a * f - c * d) / det},
          {C / det, -(a * h - b * g) / det, (a * e - b * d) / det}}};
    return true;
}
}  // namespace

extern "C" gls_status gls_dng_demosaic_params(const gls_dng_info* info, const float* xyz_rgb, int32_t camera,
                                              gls_demosaic_params* p) {
    clear_error();
    if (!info || !p) return set_error(GLS_ERR_INVALID_ARG, "NULL argument");
    if (!info->has_color_matrix1 && !info->has_color_matrix2)
        return set_error(GLS_ERR_INVALID_ARG, "the DNG has no colour matrix");
    gls_demosaic_params q{};
    q.levels = 5;
    // the camera's noise model and denoise schedule at the ISO (:48-55)
    {
        const gls_status st = calibration_fill(camera, info->iso, &q);
        if (st != GLS_OK) return st;
    }
    static const float srgb[9] = {0.4124564f, 0.3575761f, 0.1804375f, 0.2126729f, 0.7151522f,
                                  0.0721750f, 0.0193339f, 0.1191920f, 0.9503041f};
    const float* xr = xyz_rgb ? xyz_rgb : srgb;
    for (int k = 0; k < 9; k++) q.xyz_rgb[k] = xr[k];
    // unpackDNGMetadata (demosaic_utils.cpp:268-366), auto_white_balance off
    const float* cm = info->has_color_matrix2 ? info->color_matrix2 : info->color_matrix1;
    const float exposure_multiplier = float(std::pow(2.0, double(info->baseline_exposure)));
    q.black_level = info->black_level;
    q.white_level = info->white_level;
    q.exposure_multiplier = std::min(exposure_multiplier, 1.0f);
    q.bayer_pattern = bayer_of(info->cfa_pattern);
    M3 cam_xyz, xyz{};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) cam_xyz[i][j] = cm[3 * i + j], xyz[i][j] = xr[3 * i + j];
    // cam_xyz_coeff (demosaic_utils.cpp:78-101)
    const M3 cam_rgb = mul3(cam_xyz, xyz);
    float cam_white[3], pre_mul[3];
    for (int i = 0; i < 3; i++) cam_white[i] = cam_rgb[i][0] + cam_rgb[i][1] + cam_rgb[i][2];
    for (int i = 0; i < 3; i++) {
        if (!(cam_white[i] > 0.00001f)) return set_error(GLS_ERR_RANGE, "Singular Matrix");
        pre_mul[i] = 1 / cam_white[i];
    }
    M3 pm{};
    for (int i = 0; i < 3; i++) pm[i][i] = 1 / cam_white[i];
    M3 rgb_cam;
    if (!inv3(mul3(pm, cam_rgb), rgb_cam)) return set_error(GLS_ERR_RANGE, "Singular Matrix");
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) q.rgb_cam[3 * i + j] = rgb_cam[i][j];
    if (info->has_as_shot_neutral)
        for (int c = 0; c < 3; c++) pre_mul[c] = 1.0f / info->as_shot_neutral[c];
    const float mn = std::min({pre_mul[0], pre_mul[1], pre_mul[2]});
    for (int c = 0; c < 4; c++) {
        const int idx = c == 3 ? 1 : c;
        q.scale_mul[c] = float(double(std::max(exposure_multiplier, 1.0f) * (pre_mul[idx] / mn)) * 65535.0 /
                               double(q.white_level - q.black_level));
    }
    *p = q;
    return GLS_OK;
}

extern "C" int32_t gls_dng_camera(const gls_dng_info* info) {
    if (!info) return -1;
    const std::string make = info->make, model = info->model;
    if (make == "Apple" && (model == "iPhone 14 Pro" || model == "iPhone 14 Pro Max"))
        return GLS_CAMERA_IPHONE14_WIDE;  // the wide camera's calibration; other lenses fall back to it
    return -1;
}
