// ingest.cpp -- movie files to u16 frames on the host (file ingest of the
// locate path): multi-page TIFF and Olympus ETS, as the reference reads them
// (gpu-tracking/src/decoderiter.rs, execute_gpu.rs:510-542).
//
// TIFF (decoderiter.rs:9-76 through the `tiff` crate): every page of the
// file is a frame; 8- and 16-bit unsigned single-sample pages (8-bit
// values widened exactly), anything else is "Wrong bit depth".  Classic and
// BigTIFF, either byte order, strips or tiles, compression none / LZW /
// Deflate / PackBits, horizontal-differencing predictor.
//
// ETS (decoderiter.rs:78-260, MinimalETSParser): "SIS" header, "ETS"
// header with the data type and the two dimensions, then the used-chunk
// table; a chunk's coordinate 4 is its channel and coordinate 2 its frame;
// frames absent from the table are skipped.  Frames are raw little-endian
// u16 of dims[0] * dims[1] values.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>
#include <zlib.h>

#include "ingest.h"

namespace gt {

namespace {

struct File {
    int fd = -1;
    uint64_t size = 0;
    ~File() {
        if (fd >= 0) close(fd);
    }
    bool open_path(const char* path) {
        fd = ::open(path, O_RDONLY);
        if (fd < 0) return false;
        struct stat st;
        if (fstat(fd, &st) != 0) return false;
        size = (uint64_t)st.st_size;
        return true;
    }
    bool read(uint64_t off, void* dst, size_t n) const {
        if (off > size || n > size - off) return false;
        char* p = (char*)dst;
        while (n > 0) {
            const ssize_t r = ::pread(fd, p, n, (off_t)off);
            if (r <= 0) {
                if (r < 0 && errno == EINTR) continue;
                return false;
            }
            p += r;
            off += (uint64_t)r;
            n -= (size_t)r;
        }
        return true;
    }
};

// ---------------------------------------------------------------- TIFF ----

struct Page {
    uint32_t W = 0, H = 0, bits = 1, spp = 1, compression = 1, predictor = 1, planar = 1, sformat = 1;
    uint32_t rps = 0xffffffffu, tw = 0, tl = 0;
    std::vector<uint64_t> offs, counts;
};

struct Tiff {
    const File* f;
    bool le = true, big = false;
    bool u16(uint64_t off, uint32_t* v) const {
        uint8_t b[2];
        if (!f->read(off, b, 2)) return false;
        *v = le ? (uint32_t)(b[0] | b[1] << 8) : (uint32_t)(b[1] | b[0] << 8);
        return true;
    }
    bool u32(uint64_t off, uint64_t* v) const {
        uint8_t b[4];
        if (!f->read(off, b, 4)) return false;
        uint64_t x = 0;
        for (int i = 0; i < 4; ++i) x |= (uint64_t)b[le ? i : 3 - i] << (8 * i);
        *v = x;
        return true;
    }
    bool u64(uint64_t off, uint64_t* v) const {
        uint8_t b[8];
        if (!f->read(off, b, 8)) return false;
        uint64_t x = 0;
        for (int i = 0; i < 8; ++i) x |= (uint64_t)b[le ? i : 7 - i] << (8 * i);
        *v = x;
        return true;
    }
    static int type_size(uint32_t t) {
        switch (t) {
            case 1: case 2: case 6: case 7: return 1;
            case 3: case 8: return 2;
            case 4: case 9: case 11: return 4;
            case 5: case 10: case 12: case 16: case 17: case 18: return 8;
            default: return 0;
        }
    }
    uint64_t get(const uint8_t* b, int n) const {
        uint64_t x = 0;
        for (int i = 0; i < n; ++i) x |= (uint64_t)b[le ? i : n - 1 - i] << (8 * i);
        return x;
    }
    // integer values (BYTE/SHORT/LONG/LONG8) of the entry whose bytes are `e`
    bool values(const uint8_t* e, std::vector<uint64_t>* out) const {
        const uint32_t type = (uint32_t)get(e + 2, 2);
        const int ts = type_size(type);
        if (ts == 0) return false;
        const uint64_t count = big ? get(e + 4, 8) : get(e + 4, 4);
        const int inl = big ? 8 : 4;
        const uint8_t* inline_v = e + (big ? 12 : 8);
        if (count > (1ull << 28)) return false;
        std::vector<uint8_t> buf;
        const uint8_t* src = inline_v;
        if ((uint64_t)ts * count > (uint64_t)inl) {
            buf.resize((size_t)(ts * count));
            if (!f->read(get(inline_v, inl), buf.data(), buf.size())) return false;
            src = buf.data();
        }
        out->resize(count);
        for (uint64_t i = 0; i < count; ++i) {
            const uint8_t* q = src + i * ts;
            switch (type) {
                case 1: case 7: (*out)[i] = q[0]; break;
                case 3: (*out)[i] = get(q, 2); break;
                case 4: (*out)[i] = get(q, 4); break;
                case 16: case 18: (*out)[i] = get(q, 8); break;
                default: return false;
            }
        }
        return true;
    }
    // parses the IFD at `off` (one read for its entries); *next = offset of
    // the following IFD (0 at the end)
    bool ifd(uint64_t off, Page* p, uint64_t* next) const {
        uint8_t nb[8];
        const int cn = big ? 8 : 2;
        if (!f->read(off, nb, cn)) return false;
        const uint64_t n = get(nb, cn);
        if (n > 4096) return false;
        const uint64_t esz = big ? 20 : 12;
        const int nn = big ? 8 : 4;
        std::vector<uint8_t> ents((size_t)(n * esz + nn));
        if (!f->read(off + cn, ents.data(), ents.size())) return false;
        std::vector<uint64_t> v;
        for (uint64_t i = 0; i < n; ++i) {
            const uint8_t* e = ents.data() + i * esz;
            const uint32_t tag = (uint32_t)get(e, 2);
            auto one = [&](uint32_t* dst) {
                if (!values(e, &v) || v.empty()) return false;
                *dst = (uint32_t)v[0];
                return true;
            };
            bool ok = true;
            switch (tag) {
                case 256: ok = one(&p->W); break;
                case 257: ok = one(&p->H); break;
                case 258: ok = one(&p->bits); break;
                case 259: ok = one(&p->compression); break;
                case 273: case 324: ok = values(e, &p->offs); break;
                case 277: ok = one(&p->spp); break;
                case 278: ok = one(&p->rps); break;
                case 279: case 325: ok = values(e, &p->counts); break;
                case 284: ok = one(&p->planar); break;
                case 317: ok = one(&p->predictor); break;
                case 322: ok = one(&p->tw); break;
                case 323: ok = one(&p->tl); break;
                case 339: ok = one(&p->sformat); break;
                default: break;
            }
            if (!ok) return false;
        }
        *next = get(ents.data() + n * esz, nn);
        return true;
    }
};

// TIFF LZW: 9..12-bit codes, MSB first, clear 256, end 257, code width grows
// one code early.
bool lzw_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
    std::vector<uint32_t> prefix(4096);
    std::vector<uint8_t> suffix(4096), first(4096);
    std::vector<uint16_t> len(4096);
    for (int i = 0; i < 256; ++i) { prefix[i] = 0xffffffffu; suffix[i] = (uint8_t)i; first[i] = (uint8_t)i; len[i] = 1; }
    size_t pos = 0, bitpos = 0;
    int width = 9, next = 258;
    int old = -1;
    auto emit = [&](int code) -> bool {
        const int L = len[code];
        if (pos + (size_t)L > cap) return false;
        int c = code;
        for (int k = L - 1; k >= 0; --k) {
            out[pos + k] = suffix[c];
            c = (int)prefix[c];
        }
        pos += L;
        return true;
    };
    while (true) {
        if (bitpos + width > n * 8) break;
        uint32_t code = 0;
        for (int b = 0; b < width; ++b) {
            const size_t bp = bitpos + b;
            code = (code << 1) | ((in[bp >> 3] >> (7 - (bp & 7))) & 1);
        }
        bitpos += width;
        if (code == 257) break;
        if (code == 256) {
            width = 9;
            next = 258;
            old = -1;
            continue;
        }
        if (old < 0) {
            if (code > 255) return false;
            if (!emit((int)code)) return false;
            old = (int)code;
            continue;
        }
        if ((int)code < next) {
            if (!emit((int)code)) return false;
            if (next < 4096) {
                prefix[next] = (uint32_t)old; suffix[next] = first[code]; first[next] = first[old];
                len[next] = (uint16_t)(len[old] + 1);
                ++next;
            }
        } else if ((int)code == next && next < 4096) {
            prefix[next] = (uint32_t)old; suffix[next] = first[old]; first[next] = first[old];
            len[next] = (uint16_t)(len[old] + 1);
            ++next;
            if (!emit((int)code)) return false;
        } else {
            return false;
        }
        old = (int)code;
        if (next + 1 >= (1 << width) && width < 12) ++width;
    }
    if (pos < cap) std::memset(out + pos, 0, cap - pos);
    return true;
}

bool packbits_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
    size_t i = 0, o = 0;
    while (i < n && o < cap) {
        const int8_t h = (int8_t)in[i++];
        if (h >= 0) {
            const size_t k = (size_t)h + 1;
            if (i + k > n || o + k > cap) return false;
            std::memcpy(out + o, in + i, k);
            i += k;
            o += k;
        } else if (h != -128) {
            const size_t k = (size_t)(1 - h);
            if (i >= n || o + k > cap) return false;
            std::memset(out + o, in[i++], k);
            o += k;
        }
    }
    if (o < cap) std::memset(out + o, 0, cap - o);
    return true;
}

bool inflate_decode(const uint8_t* in, size_t n, uint8_t* out, size_t cap) {
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return false;
    zs.next_in = const_cast<uint8_t*>(in);
    zs.avail_in = (uInt)n;
    zs.next_out = out;
    zs.avail_out = (uInt)cap;
    const int r = inflate(&zs, Z_FINISH);
    const size_t got = cap - zs.avail_out;
    inflateEnd(&zs);
    if (r != Z_STREAM_END && r != Z_BUF_ERROR && r != Z_OK) return false;
    if (got < cap) std::memset(out + got, 0, cap - got);
    return true;
}

// One strip or tile: decompress `count` bytes at `off` into rows x cols
// samples (native u16), undoing the predictor.
bool decode_block(const File& f, const Tiff& tf, const Page& p, uint64_t off, uint64_t count, int rows, int cols,
                  std::vector<uint8_t>& raw, std::vector<uint8_t>& tmp, std::vector<uint16_t>& smp, std::string* msg) {
    const int bps = p.bits / 8;
    const size_t need = (size_t)rows * cols * bps;
    raw.resize(need);
    if (p.compression == 1) {
        if (count < need && count != 0) { *msg = "truncated strip"; return false; }
        if (!f.read(off, raw.data(), need)) { *msg = "cannot read strip"; return false; }
    } else {
        tmp.resize(count);
        if (!f.read(off, tmp.data(), count)) { *msg = "cannot read strip"; return false; }
        bool ok = false;
        if (p.compression == 5) ok = lzw_decode(tmp.data(), count, raw.data(), need);
        else if (p.compression == 8 || p.compression == 32946) ok = inflate_decode(tmp.data(), count, raw.data(), need);
        else if (p.compression == 32773) ok = packbits_decode(tmp.data(), count, raw.data(), need);
        else { *msg = "TIFF compression " + std::to_string(p.compression) + " is not supported"; return false; }
        if (!ok) { *msg = "corrupt compressed strip"; return false; }
    }
    smp.resize((size_t)rows * cols);
    if (bps == 1) {
        for (size_t i = 0; i < smp.size(); ++i) smp[i] = raw[i];
    } else {
        for (size_t i = 0; i < smp.size(); ++i)
            smp[i] = tf.le ? (uint16_t)(raw[2 * i] | raw[2 * i + 1] << 8) : (uint16_t)(raw[2 * i + 1] | raw[2 * i] << 8);
    }
    if (p.predictor == 2) {
        const uint32_t mask = bps == 1 ? 0xffu : 0xffffu;
        for (int r = 0; r < rows; ++r) {
            uint16_t* row = smp.data() + (size_t)r * cols;
            for (int c = 1; c < cols; ++c) row[c] = (uint16_t)((row[c] + row[c - 1]) & mask);
        }
    } else if (p.predictor != 1) {
        *msg = "TIFF predictor " + std::to_string(p.predictor) + " is not supported";
        return false;
    }
    return true;
}

bool decode_page(const File& f, const Tiff& tf, const Page& p, uint16_t* out, std::string* msg) {
    std::vector<uint8_t> raw, tmp;
    std::vector<uint16_t> smp;
    const int W = (int)p.W, H = (int)p.H;
    if (p.tw && p.tl) {
        const int tw = (int)p.tw, tl = (int)p.tl;
        const int nx = (W + tw - 1) / tw, ny = (H + tl - 1) / tl;
        if (p.offs.size() < (size_t)nx * ny) { *msg = "missing tile offsets"; return false; }
        for (int ty = 0; ty < ny; ++ty)
            for (int tx = 0; tx < nx; ++tx) {
                const size_t k = (size_t)ty * nx + tx;
                const uint64_t cnt = k < p.counts.size() ? p.counts[k] : 0;
                if (!decode_block(f, tf, p, p.offs[k], cnt, tl, tw, raw, tmp, smp, msg)) return false;
                for (int r = 0; r < tl && ty * tl + r < H; ++r) {
                    const int cw = std::min(tw, W - tx * tw);
                    std::memcpy(out + (size_t)(ty * tl + r) * W + tx * tw, smp.data() + (size_t)r * tw,
                                sizeof(uint16_t) * cw);
                }
            }
        return true;
    }
    const int rps = (int)std::min<uint32_t>(p.rps, (uint32_t)H);
    const int ns = (H + rps - 1) / rps;
    if (p.offs.size() < (size_t)ns) { *msg = "missing strip offsets"; return false; }
    if (p.compression == 1 && p.bits == 16 && tf.le && p.predictor == 1) {
        // raw little-endian samples: straight into the frame
        for (int s = 0; s < ns; ++s) {
            const int rows = std::min(rps, H - s * rps);
            if (!f.read(p.offs[s], out + (size_t)s * rps * W, sizeof(uint16_t) * (size_t)rows * W)) {
                *msg = "cannot read strip";
                return false;
            }
        }
        return true;
    }
    for (int s = 0; s < ns; ++s) {
        const int rows = std::min(rps, H - s * rps);
        const uint64_t cnt = (size_t)s < p.counts.size() ? p.counts[s] : 0;
        if (!decode_block(f, tf, p, p.offs[s], cnt, rows, W, raw, tmp, smp, msg)) return false;
        std::memcpy(out + (size_t)s * rps * W, smp.data(), sizeof(uint16_t) * (size_t)rows * W);
    }
    return true;
}

bool tiff_pages(const File& f, Tiff* tf, std::vector<Page>* pages, std::string* msg) {
    uint8_t h[16];
    if (!f.read(0, h, 8)) { *msg = "not a TIFF file"; return false; }
    if (h[0] == 'I' && h[1] == 'I') tf->le = true;
    else if (h[0] == 'M' && h[1] == 'M') tf->le = false;
    else { *msg = "not a TIFF file"; return false; }
    uint32_t magic = 0;
    uint64_t off = 0;
    if (!tf->u16(2, &magic)) { *msg = "not a TIFF file"; return false; }
    if (magic == 42) {
        tf->big = false;
        if (!tf->u32(4, &off)) { *msg = "truncated TIFF header"; return false; }
    } else if (magic == 43) {
        tf->big = true;
        if (!tf->u64(8, &off)) { *msg = "truncated BigTIFF header"; return false; }
    } else {
        *msg = "not a TIFF file";
        return false;
    }
    std::map<uint64_t, int> seen;
    while (off != 0) {
        if (seen.count(off) || pages->size() > (1u << 24)) { *msg = "looping IFD chain"; return false; }
        seen[off] = 1;
        Page p;
        uint64_t next = 0;
        if (!tf->ifd(off, &p, &next)) { *msg = "corrupt IFD"; return false; }
        pages->push_back(p);
        off = next;
    }
    if (pages->empty()) { *msg = "TIFF without pages"; return false; }
    return true;
}

// ----------------------------------------------------------------- ETS ----

struct Ets {
    uint32_t dtype = 0;
    uint32_t dims[2] = {0, 0};
    std::map<uint64_t, std::vector<int64_t>> offsets;  // channel -> frame offsets (-1 = absent)
};

bool rd32(const File& f, uint64_t off, uint32_t* v) {
    uint8_t b[4];
    if (!f.read(off, b, 4)) return false;
    *v = (uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24;
    return true;
}
bool rd64(const File& f, uint64_t off, uint64_t* v) {
    uint32_t lo, hi;
    if (!rd32(f, off, &lo) || !rd32(f, off + 4, &hi)) return false;
    *v = (uint64_t)hi << 32 | lo;
    return true;
}

// decoderiter.rs:133-183
bool ets_parse(const File& f, Ets* e, std::string* msg) {
    char m[4];
    if (!f.read(0, m, 4) || std::memcmp(m, "SIS\0", 4) != 0) { *msg = "not an ETS file (no SIS header)"; return false; }
    uint32_t ndim, nused;
    uint64_t add_off, used_off;
    if (!rd32(f, 12, &ndim) || !rd64(f, 16, &add_off) || !rd64(f, 32, &used_off) || !rd32(f, 40, &nused)) {
        *msg = "truncated ETS header";
        return false;
    }
    if (ndim < 5 || ndim > 64) { *msg = "ETS chunk coordinates have " + std::to_string(ndim) + " dimensions"; return false; }
    if (!f.read(add_off, m, 4) || std::memcmp(m, "ETS\0", 4) != 0) { *msg = "not an ETS file (no ETS header)"; return false; }
    if (!rd32(f, add_off + 8, &e->dtype) || !rd32(f, add_off + 28, &e->dims[0]) || !rd32(f, add_off + 32, &e->dims[1])) {
        *msg = "truncated ETS header";
        return false;
    }
    uint64_t pos = used_off;
    std::vector<uint32_t> coord(ndim);
    for (uint32_t c = 0; c < nused; ++c) {
        pos += 4;
        for (uint32_t d = 0; d < ndim; ++d) {
            if (!rd32(f, pos, &coord[d])) { *msg = "truncated ETS chunk table"; return false; }
            pos += 4;
        }
        uint64_t o;
        if (!rd64(f, pos, &o)) { *msg = "truncated ETS chunk table"; return false; }
        pos += 8 + 8;
        // decoderiter.rs:163-174, including its handling of a repeated
        // last frame index (appended as one more frame)
        std::vector<int64_t>& v = e->offsets[coord[4]];
        const size_t c2 = coord[2];
        if (c2 + 1 == v.size()) {
            v.push_back((int64_t)o);
        } else if (c2 + 1 > v.size()) {
            v.resize(c2 + 1, -1);
            v[c2] = (int64_t)o;
        } else {
            v[c2] = (int64_t)o;
        }
    }
    return true;
}

bool ends_with(const std::string& s, const char* ext) {
    const size_t n = std::strlen(ext);
    if (s.size() < n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)s[s.size() - n + i]) != ext[i]) return false;
    return true;
}

}  // namespace

struct MovieFile::Impl {
    File f;
    bool ets = false;
    Tiff tf;
    std::vector<Page> pages;
    std::vector<int64_t> frames;  // ETS frame offsets of the channel, absent ones dropped
};

MovieFile::MovieFile() : impl(new Impl) {}
MovieFile::~MovieFile() { delete impl; }

int MovieFile::open(const char* path, bool has_channel, uint32_t channel, std::string* msg) {
    if (!path || !impl->f.open_path(path)) {
        *msg = std::string("Could not open file ") + (path ? path : "(null)");
        return 1;
    }
    const std::string p(path);
    if (ends_with(p, ".tif") || ends_with(p, ".tiff")) {
        impl->tf.f = &impl->f;
        if (!tiff_pages(impl->f, &impl->tf, &impl->pages, msg)) return 1;
        const Page& p0 = impl->pages[0];
        H = (int)p0.H;
        W = (int)p0.W;
        for (const Page& pg : impl->pages) {
            if (pg.bits != 8 && pg.bits != 16) { *msg = "Wrong bit depth"; return 2; }
            if (pg.spp != 1 || pg.sformat != 1) { *msg = "Wrong bit depth"; return 2; }
            if (pg.W != p0.W || pg.H != p0.H) { *msg = "pages of different sizes"; return 1; }
        }
        T = (int)impl->pages.size();
        return 0;
    }
    if (ends_with(p, ".ets")) {
        impl->ets = true;
        Ets e;
        if (!ets_parse(impl->f, &e, msg)) return 1;
        if (e.dtype != 4) {
            *msg = "ETS data type " + std::to_string(e.dtype) + " is not supported (u16 frames only)";
            return 2;
        }
        const uint64_t ch = has_channel ? channel : 0;
        auto it = e.offsets.find(ch);
        if (it == e.offsets.end()) { *msg = "ETS file has no channel " + std::to_string(ch); return 1; }
        for (int64_t o : it->second)
            if (o >= 0) impl->frames.push_back(o);
        // execute_gpu.rs:527: dims[0] rows, dims[1] columns
        H = (int)e.dims[0];
        W = (int)e.dims[1];
        T = (int)impl->frames.size();
        if (T == 0) { *msg = "ETS channel without frames"; return 1; }
        return 0;
    }
    *msg = "File extension '" + p.substr(p.find_last_of('.') == std::string::npos ? p.size() : p.find_last_of('.') + 1) +
           "' not supported";
    return 1;
}

int MovieFile::read_frame(int t, uint16_t* out, std::string* msg) const {
    if (t < 0 || t >= T) { *msg = "frame out of range"; return 1; }
    if (impl->ets) {
        if (!impl->f.read((uint64_t)impl->frames[t], out, sizeof(uint16_t) * (size_t)H * W)) {
            *msg = "truncated ETS frame";
            return 1;
        }
        return 0;
    }
    return decode_page(impl->f, impl->tf, impl->pages[t], out, msg) ? 0 : 1;
}

int ets_channels(const char* path, std::vector<std::pair<uint32_t, int>>* chans, uint32_t dims[2], std::string* msg) {
    File f;
    if (!path || !f.open_path(path)) { *msg = std::string("Could not open file ") + (path ? path : "(null)"); return 1; }
    Ets e;
    if (!ets_parse(f, &e, msg)) return 1;
    dims[0] = e.dims[0];
    dims[1] = e.dims[1];
    for (auto& kv : e.offsets) {
        int n = 0;
        for (int64_t o : kv.second) n += o >= 0;
        chans->push_back({(uint32_t)kv.first, n});
    }
    return 0;
}

}  // namespace gt
