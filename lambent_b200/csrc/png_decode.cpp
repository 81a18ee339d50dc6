// png_decode.cpp - PNG decoding for TextureLoader::load / load_from_bytes (src/textures.rs:25-38),
// which the reference delegates to image 0.25.6 (image::load_from_memory(..).to_rgba8()).
// Implements zlib/DEFLATE (RFC 1950/1951) and PNG (RFC 2083) for non-interlaced images of
// colour types 0, 2, 3, 4, 6 at bit depth 8 (and 16, reduced to 8 bits with rounding, and 1/2/4
// for grey and palette).  Output: RGBA8, row-major, top row first.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

namespace lam {
namespace {

struct BitReader {
    const uint8_t* p;
    size_t n, pos = 0;
    uint32_t bitbuf = 0;
    int bitcnt = 0;
    bool err = false;
    int bit() {
        if (bitcnt == 0) {
            if (pos >= n) { err = true; return 0; }
            bitbuf = p[pos++];
            bitcnt = 8;
        }
        int b = bitbuf & 1;
        bitbuf >>= 1;
        bitcnt--;
        return b;
    }
    uint32_t bits(int k) {
        uint32_t v = 0;
        for (int i = 0; i < k; ++i) v |= (uint32_t)bit() << i;
        return v;
    }
    void align() { bitcnt = 0; }
};

struct Huffman {
    uint16_t count[16] = {0};
    uint16_t symbol[320] = {0};
    bool build(const uint8_t* lengths, int n) {
        std::memset(count, 0, sizeof(count));
        for (int i = 0; i < n; ++i) count[lengths[i]]++;
        count[0] = 0;
        int left = 1;
        for (int len = 1; len < 16; ++len) {
            left <<= 1;
            left -= count[len];
            if (left < 0) return false;
        }
        uint16_t offs[16];
        offs[1] = 0;
        for (int len = 1; len < 15; ++len) offs[len + 1] = offs[len] + count[len];
        for (int i = 0; i < n; ++i)
            if (lengths[i]) symbol[offs[lengths[i]]++] = (uint16_t)i;
        return true;
    }
    int decode(BitReader& br) const {
        int code = 0, first = 0, index = 0;
        for (int len = 1; len < 16; ++len) {
            code |= br.bit();
            int c = count[len];
            if (code - c < first) return symbol[index + (code - first)];
            index += c;
            first += c;
            first <<= 1;
            code <<= 1;
            if (br.err) return -1;
        }
        return -1;
    }
};

const uint16_t LBASE[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31, 35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t LEXT[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t DBASE[30] = {1, 2, 3, 4, 5, 7, 9, 13, 17, 25, 33, 49, 65, 97, 129, 193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t DEXT[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

bool inflate_block(BitReader& br, const Huffman& lit, const Huffman& dist, std::vector<uint8_t>& out) {
    for (;;) {
        int sym = lit.decode(br);
        if (sym < 0 || br.err) return false;
        if (sym < 256) {
            out.push_back((uint8_t)sym);
        } else if (sym == 256) {
            return true;
        } else {
            sym -= 257;
            if (sym >= 29) return false;
            size_t len = LBASE[sym] + br.bits(LEXT[sym]);
            int ds = dist.decode(br);
            if (ds < 0 || ds >= 30) return false;
            size_t d = DBASE[ds] + br.bits(DEXT[ds]);
            if (d > out.size()) return false;
            size_t start = out.size() - d;
            for (size_t i = 0; i < len; ++i) out.push_back(out[start + i]);
        }
    }
}

bool inflate(const uint8_t* p, size_t n, std::vector<uint8_t>& out) {
    if (n < 2) return false;
    if ((p[0] & 0x0F) != 8 || ((p[0] << 8) | p[1]) % 31 != 0 || (p[1] & 0x20)) return false;
    BitReader br{p + 2, n - 2};
    int final_block = 0;
    do {
        final_block = br.bit();
        int type = (int)br.bits(2);
        if (br.err) return false;
        if (type == 0) {
            br.align();
            if (br.pos + 4 > br.n) return false;
            uint32_t len = br.p[br.pos] | (br.p[br.pos + 1] << 8);
            uint32_t nlen = br.p[br.pos + 2] | (br.p[br.pos + 3] << 8);
            br.pos += 4;
            if ((len ^ 0xFFFFu) != nlen || br.pos + len > br.n) return false;
            out.insert(out.end(), br.p + br.pos, br.p + br.pos + len);
            br.pos += len;
        } else if (type == 1) {
            uint8_t l[288], d[30];
            for (int i = 0; i < 144; ++i) l[i] = 8;
            for (int i = 144; i < 256; ++i) l[i] = 9;
            for (int i = 256; i < 280; ++i) l[i] = 7;
            for (int i = 280; i < 288; ++i) l[i] = 8;
            for (int i = 0; i < 30; ++i) d[i] = 5;
            Huffman lit, dist;
            lit.build(l, 288);
            dist.build(d, 30);
            if (!inflate_block(br, lit, dist, out)) return false;
        } else if (type == 2) {
            int hlit = (int)br.bits(5) + 257, hdist = (int)br.bits(5) + 1, hclen = (int)br.bits(4) + 4;
            static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
            uint8_t cl[19] = {0};
            for (int i = 0; i < hclen; ++i) cl[order[i]] = (uint8_t)br.bits(3);
            Huffman clh;
            if (!clh.build(cl, 19)) return false;
            uint8_t lens[320] = {0};
            int idx = 0;
            while (idx < hlit + hdist) {
                int sym = clh.decode(br);
                if (sym < 0 || br.err) return false;
                if (sym < 16) {
                    lens[idx++] = (uint8_t)sym;
                } else {
                    int rep = 0;
                    uint8_t val = 0;
                    if (sym == 16) {
                        if (idx == 0) return false;
                        val = lens[idx - 1];
                        rep = 3 + (int)br.bits(2);
                    } else if (sym == 17) {
                        rep = 3 + (int)br.bits(3);
                    } else {
                        rep = 11 + (int)br.bits(7);
                    }
                    if (idx + rep > hlit + hdist) return false;
                    while (rep--) lens[idx++] = val;
                }
            }
            Huffman lit, dist;
            if (!lit.build(lens, hlit) || !dist.build(lens + hlit, hdist)) return false;
            if (!inflate_block(br, lit, dist, out)) return false;
        } else {
            return false;
        }
    } while (!final_block);
    return true;
}

uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

int paeth(int a, int b, int c) {
    int p = a + b - c;
    int pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
    if (pa <= pb && pa <= pc) return a;
    if (pb <= pc) return b;
    return c;
}

}  // namespace

// Returns true on success; on failure writes a reason to *why.
bool decode_png(const uint8_t* data, size_t n, std::vector<uint8_t>* rgba, uint32_t* w_out, uint32_t* h_out,
                std::string* why) {
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (n < 8 || std::memcmp(data, sig, 8) != 0) { *why = "not a PNG file"; return false; }
    size_t pos = 8;
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, palette, trns;
    bool seen_end = false;
    while (pos + 12 <= n) {
        uint32_t len = be32(data + pos);
        const uint8_t* type = data + pos + 4;
        if (pos + 12 + (size_t)len > n) { *why = "truncated chunk"; return false; }
        const uint8_t* body = data + pos + 8;
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) { *why = "bad IHDR"; return false; }
            w = be32(body);
            h = be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (!std::memcmp(type, "PLTE", 4)) {
            palette.assign(body, body + len);
        } else if (!std::memcmp(type, "tRNS", 4)) {
            trns.assign(body, body + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), body, body + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            seen_end = true;
            break;
        }
        pos += 12 + (size_t)len;
    }
    if (!seen_end || w == 0 || h == 0) { *why = "missing IHDR/IEND"; return false; }
    if (interlace) { *why = "interlaced PNG is not supported"; return false; }
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: *why = "unknown colour type"; return false;
    }
    bool depth_ok = depth == 8 || (depth == 16 && ctype != 3) || ((depth == 1 || depth == 2 || depth == 4) && (ctype == 0 || ctype == 3));
    if (!depth_ok) { *why = "unsupported bit depth"; return false; }
    if ((uint64_t)w * h > (1ull << 28)) { *why = "image too large"; return false; }
    size_t bpp_bits = (size_t)channels * depth;
    size_t stride = ((size_t)w * bpp_bits + 7) / 8;
    size_t bpp = std::max<size_t>(1, bpp_bits / 8);
    std::vector<uint8_t> raw;
    raw.reserve((stride + 1) * h);
    if (!inflate(idat.data(), idat.size(), raw)) { *why = "corrupt zlib stream"; return false; }
    if (raw.size() < (stride + 1) * h) { *why = "short image data"; return false; }
    std::vector<uint8_t> cur(stride), prev(stride, 0);
    rgba->assign((size_t)w * h * 4, 0);
    for (uint32_t y = 0; y < h; ++y) {
        const uint8_t* line = raw.data() + y * (stride + 1);
        uint8_t ft = line[0];
        for (size_t i = 0; i < stride; ++i) {
            int x = line[1 + i];
            int a = i >= bpp ? cur[i - bpp] : 0;
            int b = prev[i];
            int c = i >= bpp ? prev[i - bpp] : 0;
            switch (ft) {
                case 0: break;
                case 1: x += a; break;
                case 2: x += b; break;
                case 3: x += (a + b) / 2; break;
                case 4: x += paeth(a, b, c); break;
                default: *why = "bad filter type"; return false;
            }
            cur[i] = (uint8_t)x;
        }
        for (uint32_t xpix = 0; xpix < w; ++xpix) {
            uint8_t* o = rgba->data() + 4 * ((size_t)y * w + xpix);
            auto sample = [&](int ch) -> uint32_t {
                if (depth == 8) return cur[(size_t)xpix * channels + ch];
                if (depth == 16) {
                    uint32_t v = ((uint32_t)cur[2 * ((size_t)xpix * channels + ch)] << 8) | cur[2 * ((size_t)xpix * channels + ch) + 1];
                    return (v * 255u + 32767u) / 65535u;
                }
                size_t bitpos = (size_t)xpix * depth;
                uint32_t v = (cur[bitpos / 8] >> (8 - depth - (bitpos % 8))) & ((1u << depth) - 1u);
                return v;
            };
            if (ctype == 3) {
                uint32_t i = sample(0);
                if (3 * i + 2 >= palette.size()) { *why = "palette index out of range"; return false; }
                o[0] = palette[3 * i];
                o[1] = palette[3 * i + 1];
                o[2] = palette[3 * i + 2];
                o[3] = i < trns.size() ? trns[i] : 255;
            } else if (ctype == 0 || ctype == 4) {
                uint32_t g = sample(0);
                if (depth < 8) g = g * 255u / ((1u << depth) - 1u);
                o[0] = o[1] = o[2] = (uint8_t)g;
                o[3] = ctype == 4 ? (uint8_t)sample(1) : 255;
            } else {
                o[0] = (uint8_t)sample(0);
                o[1] = (uint8_t)sample(1);
                o[2] = (uint8_t)sample(2);
                o[3] = ctype == 6 ? (uint8_t)sample(3) : 255;
            }
        }
        std::swap(cur, prev);
    }
    *w_out = w;
    *h_out = h;
    return true;
}

}  // namespace lam
