// Image decoding for the command-line driver: what cv::imread(path,
// IMREAD_COLOR) returns for the inputs of HPM-MVS++ (main.cpp:123-126,
// 212-213), as 8-bit BGR.  The format is sniffed from the content, as imread
// does, so PNG bytes in a file named .jpg are read as PNG.
//
//   PNG  (ISO/IEC 15948): colour types 0/2/3/4/6, bit depths 1-16, no
//        interlace; zlib inflate, the five row filters; 16-bit samples keep
//        their high byte, alpha is dropped, grey is replicated.  Lossless, so
//        the result equals imread's.
//   JPEG (ITU-T T.81 baseline and extended sequential Huffman, 8-bit): any
//        sampling factors up to 4x4, restart intervals; a floating-point
//        inverse DCT, chroma upsampled by the triangle filter (2:1 ratios) or
//        by replication (other ratios), JFIF YCbCr to
//        RGB.  libjpeg's integer IDCT and rounding differ in the last grey
//        level, so the result is within a few levels of imread's, not equal.
//        Progressive and arithmetic-coded files are rejected.
#include "hpm_host.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

thread_local std::string g_error;

int fail(const std::string& msg) {
    g_error = msg;
    return -1;
}

// ------------------------------------------------------------------ PNG

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

int decode_png(const uint8_t* d, size_t n, std::vector<uint8_t>& bgr, int& W, int& H) {
    size_t pos = 8;
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<uint8_t> idat, plte;
    bool have_end = false;
    while (pos + 12 <= n && !have_end) {
        const uint32_t len = be32(d + pos);
        const uint8_t* type = d + pos + 4;
        if (pos + 12 + (size_t)len > n) return fail("PNG: truncated chunk");
        const uint8_t* body = d + pos + 8;
        if (!std::memcmp(type, "IHDR", 4)) {
            if (len < 13) return fail("PNG: short IHDR");
            w = be32(body); h = be32(body + 4);
            depth = body[8]; ctype = body[9]; interlace = body[12];
        } else if (!std::memcmp(type, "PLTE", 4)) {
            plte.assign(body, body + len);
        } else if (!std::memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), body, body + len);
        } else if (!std::memcmp(type, "IEND", 4)) {
            have_end = true;
        }
        pos += 12 + len;
    }
    if (w == 0 || h == 0 || w > (1u << 16) || h > (1u << 16)) return fail("PNG: bad size");
    if (interlace) return fail("PNG: interlaced files are not supported");
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: return fail("PNG: bad colour type");
    }
    if (!(depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) return fail("PNG: bad bit depth");
    if ((ctype == 2 || ctype == 4 || ctype == 6) && depth < 8) return fail("PNG: bad bit depth for colour type");
    if (ctype == 3 && (depth == 16 || plte.size() < 3)) return fail("PNG: bad palette");
    const size_t bpp_bits = (size_t)channels * depth;
    const size_t stride = (w * bpp_bits + 7) / 8;
    const size_t bpp = std::max<size_t>(1, bpp_bits / 8);
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf raw_len = (uLongf)raw.size();
    if (uncompress(raw.data(), &raw_len, idat.data(), (uLong)idat.size()) != Z_OK || raw_len != raw.size())
        return fail("PNG: corrupt image data");
    std::vector<uint8_t> prev(stride, 0), cur(stride);
    bgr.resize((size_t)w * h * 3);
    for (uint32_t y = 0; y < h; ++y) {
        const uint8_t* line = raw.data() + y * (stride + 1);
        const int filter = line[0];
        for (size_t i = 0; i < stride; ++i) {
            const int x = line[1 + i];
            const int a = i >= bpp ? cur[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
            int v;
            switch (filter) {
                case 0: v = x; break;
                case 1: v = x + a; break;
                case 2: v = x + b; break;
                case 3: v = x + ((a + b) >> 1); break;
                case 4: v = x + paeth(a, b, c); break;
                default: return fail("PNG: bad filter type");
            }
            cur[i] = (uint8_t)v;
        }
        uint8_t* out = bgr.data() + (size_t)y * w * 3;
        for (uint32_t x = 0; x < w; ++x) {
            auto sample = [&](int ch) -> int {  // 8-bit value of channel ch of pixel x
                if (depth == 16) return cur[(x * channels + ch) * 2];
                if (depth == 8) return cur[x * channels + ch];
                const size_t bit = (size_t)x * depth;
                const int v = (cur[bit >> 3] >> (8 - depth - (bit & 7))) & ((1 << depth) - 1);
                return ctype == 3 ? v : v * 255 / ((1 << depth) - 1);
            };
            int r, g, b;
            if (ctype == 3) {
                const int idx = sample(0);
                if ((size_t)idx * 3 + 2 >= plte.size()) return fail("PNG: palette index out of range");
                r = plte[idx * 3]; g = plte[idx * 3 + 1]; b = plte[idx * 3 + 2];
            } else if (channels <= 2) {
                r = g = b = sample(0);
            } else {
                r = sample(0); g = sample(1); b = sample(2);
            }
            out[3 * x] = (uint8_t)b; out[3 * x + 1] = (uint8_t)g; out[3 * x + 2] = (uint8_t)r;
        }
        std::swap(prev, cur);
    }
    W = (int)w;
    H = (int)h;
    return 0;
}

// ------------------------------------------------------------------ JPEG

const int kZigzag[64] = { 0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                          41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                          30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63 };

struct Huffman {
    // canonical code table: for each length, first code and index of its first symbol
    int mincode[17], maxcode[18], valptr[17];
    uint8_t vals[256];
    bool present = false;
};

struct Component {
    int id, h, v, tq, td, ta;
    int bw, bh;                 // blocks per line / column in the padded plane
    std::vector<uint8_t> plane; // decoded samples, bw*8 x bh*8
    int dc_pred;
};

class Jpeg {
public:
    Jpeg(const uint8_t* d, size_t n) : d_(d), n_(n) {}
    int decode(std::vector<uint8_t>& bgr, int& W, int& H);

private:
    const uint8_t* d_;
    size_t n_;
    size_t pos_ = 0;
    uint16_t q_[4][64] = {};
    Huffman dc_[4], ac_[4];
    std::vector<Component> comps_;
    int width_ = 0, height_ = 0, hmax_ = 1, vmax_ = 1, restart_ = 0;
    // entropy reader
    uint32_t bitbuf_ = 0;
    int bitcnt_ = 0;
    bool marker_hit_ = false;

    int read_u16(size_t at) const { return (d_[at] << 8) | d_[at + 1]; }
    int fill_bit() {
        if (bitcnt_ == 0) {
            int byte = 0;
            if (!marker_hit_ && pos_ < n_) {
                byte = d_[pos_];
                if (byte == 0xFF) {
                    const int next = pos_ + 1 < n_ ? d_[pos_ + 1] : 0;
                    if (next == 0x00) { pos_ += 2; }
                    else { marker_hit_ = true; byte = 0; }
                } else {
                    ++pos_;
                }
            }
            bitbuf_ = (uint32_t)byte;
            bitcnt_ = 8;
        }
        --bitcnt_;
        return (bitbuf_ >> bitcnt_) & 1;
    }
    int receive(int s) {
        int v = 0;
        for (int i = 0; i < s; ++i) v = (v << 1) | fill_bit();
        return v;
    }
    static int extend(int v, int s) { return (s > 0 && v < (1 << (s - 1))) ? v - (1 << s) + 1 : v; }
    int decode_huff(const Huffman& hf) {
        int code = fill_bit();
        for (int l = 1; l <= 16; ++l) {
            if (code <= hf.maxcode[l]) return hf.vals[hf.valptr[l] + code - hf.mincode[l]];
            code = (code << 1) | fill_bit();
        }
        return -1;
    }
    int build_huffman(Huffman& hf, const uint8_t* counts, const uint8_t* symbols, int total) {
        if (total > 256) return fail("JPEG: Huffman table too large");
        std::memcpy(hf.vals, symbols, total);
        int code = 0, k = 0;
        for (int l = 1; l <= 16; ++l) {
            hf.valptr[l] = k;
            hf.mincode[l] = code;
            code += counts[l - 1];
            k += counts[l - 1];
            hf.maxcode[l] = counts[l - 1] ? code - 1 : -1;
            code <<= 1;
        }
        hf.maxcode[17] = 0x7fffffff;
        hf.present = true;
        return 0;
    }
    int decode_block(Component& c, int16_t coef[64]);
    int decode_scan();
    void reset_entropy() {
        bitcnt_ = 0;
        marker_hit_ = false;
        for (auto& c : comps_) c.dc_pred = 0;
    }
};

int Jpeg::decode_block(Component& c, int16_t coef[64]) {
    std::memset(coef, 0, 64 * sizeof(int16_t));
    const Huffman& dc = dc_[c.td];
    const Huffman& ac = ac_[c.ta];
    if (!dc.present || !ac.present) return fail("JPEG: missing Huffman table");
    const int t = decode_huff(dc);
    if (t < 0 || t > 15) return fail("JPEG: corrupt DC code");
    const int diff = t ? extend(receive(t), t) : 0;
    c.dc_pred += diff;
    coef[0] = (int16_t)(c.dc_pred * q_[c.tq][0]);
    for (int k = 1; k < 64;) {
        const int rs = decode_huff(ac);
        if (rs < 0) return fail("JPEG: corrupt AC code");
        const int r = rs >> 4, s = rs & 15;
        if (s == 0) {
            if (r != 15) break;  // end of block
            k += 16;
            continue;
        }
        k += r;
        if (k > 63) return fail("JPEG: coefficient index out of range");
        coef[kZigzag[k]] = (int16_t)(extend(receive(s), s) * q_[c.tq][k]);
        ++k;
    }
    return 0;
}

// Separable inverse DCT in double precision (T.81 A.3.3), level shift and clamp.
void idct_block(const int16_t in[64], uint8_t* out, int stride) {
    static double cosines[8][8];
    static bool init = false;
    if (!init) {
        for (int x = 0; x < 8; ++x)
            for (int u = 0; u < 8; ++u)
                cosines[x][u] = (u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * 3.14159265358979323846 / 16);
        init = true;
    }
    double tmp[64];
    for (int y = 0; y < 8; ++y)      // rows of the output: transform along v
        for (int u = 0; u < 8; ++u) {
            double s = 0;
            for (int v = 0; v < 8; ++v) s += cosines[y][v] * in[v * 8 + u];
            tmp[y * 8 + u] = s / 2;
        }
    for (int y = 0; y < 8; ++y)
        for (int x = 0; x < 8; ++x) {
            double s = 0;
            for (int u = 0; u < 8; ++u) s += cosines[x][u] * tmp[y * 8 + u];
            const long v = std::lround(s / 2 + 128.0);
            out[y * stride + x] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
        }
}

int Jpeg::decode_scan() {
    const int mcu_w = 8 * hmax_, mcu_h = 8 * vmax_;
    const int mcus_x = (width_ + mcu_w - 1) / mcu_w, mcus_y = (height_ + mcu_h - 1) / mcu_h;
    const bool single = comps_.size() == 1;
    reset_entropy();
    int16_t coef[64];
    int until_restart = restart_;
    auto handle_restart = [&]() -> int {
        if (!restart_) return 0;
        if (until_restart == 0) {
            // skip to the RSTn marker
            while (pos_ + 1 < n_ && !(d_[pos_] == 0xFF && d_[pos_ + 1] >= 0xD0 && d_[pos_ + 1] <= 0xD7)) ++pos_;
            if (pos_ + 1 >= n_) return fail("JPEG: missing restart marker");
            pos_ += 2;
            reset_entropy();
            until_restart = restart_;
        }
        --until_restart;
        return 0;
    };
    if (single) {
        // a single-component scan is not interleaved: blocks in raster order over the component
        Component& c = comps_[0];
        const int bx_n = (width_ * c.h / hmax_ + 7) / 8, by_n = (height_ * c.v / vmax_ + 7) / 8;
        for (int by = 0; by < by_n; ++by)
            for (int bx = 0; bx < bx_n; ++bx) {
                if (handle_restart()) return -1;
                if (decode_block(c, coef)) return -1;
                idct_block(coef, c.plane.data() + (size_t)by * 8 * c.bw * 8 + bx * 8, c.bw * 8);
            }
        return 0;
    }
    for (int my = 0; my < mcus_y; ++my)
        for (int mx = 0; mx < mcus_x; ++mx) {
            if (handle_restart()) return -1;
            for (auto& c : comps_)
                for (int v = 0; v < c.v; ++v)
                    for (int h = 0; h < c.h; ++h) {
                        if (decode_block(c, coef)) return -1;
                        const int bx = mx * c.h + h, by = my * c.v + v;
                        idct_block(coef, c.plane.data() + (size_t)by * 8 * c.bw * 8 + bx * 8, c.bw * 8);
                    }
        }
    return 0;
}

int Jpeg::decode(std::vector<uint8_t>& bgr, int& W, int& H) {
    pos_ = 2;
    bool frame = false;
    while (pos_ + 4 <= n_) {
        if (d_[pos_] != 0xFF) { ++pos_; continue; }
        const int marker = d_[pos_ + 1];
        if (marker == 0xFF) { ++pos_; continue; }
        if (marker == 0xD9) break;  // EOI
        if (marker == 0xD8 || (marker >= 0xD0 && marker <= 0xD7)) { pos_ += 2; continue; }
        const int len = read_u16(pos_ + 2);
        const size_t seg = pos_ + 4;
        if (seg + len - 2 > n_ || len < 2) return fail("JPEG: truncated segment");
        if (marker == 0xDB) {  // DQT
            const size_t end = seg + len - 2;
            size_t p = seg;
            while (p < end) {
                const int pq = d_[p] >> 4, tq = d_[p] & 15;
                if (tq > 3 || pq > 1) return fail("JPEG: bad quantisation table id or precision");
                if (p + 1 + 64 * (pq + 1) > end) return fail("JPEG: truncated quantisation table");
                ++p;
                for (int k = 0; k < 64; ++k) {
                    q_[tq][k] = pq ? (uint16_t)read_u16(p + 2 * k) : d_[p + k];
                }
                p += pq ? 128 : 64;
            }
        } else if (marker == 0xC4) {  // DHT
            const size_t end = seg + len - 2;
            size_t p = seg;
            while (p < end) {
                const int tc = d_[p] >> 4, th = d_[p] & 15;
                if (th > 3 || tc > 1) return fail("JPEG: bad Huffman table id");
                if (p + 17 > end) return fail("JPEG: truncated Huffman table");
                int total = 0;
                for (int i = 0; i < 16; ++i) total += d_[p + 1 + i];
                if (p + 17 + (size_t)total > end) return fail("JPEG: truncated Huffman table");
                if (build_huffman(tc ? ac_[th] : dc_[th], d_ + p + 1, d_ + p + 17, total)) return -1;
                p += 17 + total;
            }
        } else if (marker == 0xC0 || marker == 0xC1) {  // SOF0 / SOF1
            if (frame) return fail("JPEG: more than one frame header");
            if (len - 2 < 6) return fail("JPEG: truncated frame header");
            if (d_[seg] != 8) return fail("JPEG: only 8-bit samples are supported");
            height_ = read_u16(seg + 1);
            width_ = read_u16(seg + 3);
            const int nc = d_[seg + 5];
            if (width_ <= 0 || height_ <= 0 || (nc != 1 && nc != 3)) return fail("JPEG: unsupported frame");
            if (6 + 3 * nc > len - 2) return fail("JPEG: truncated frame header");
            comps_.resize(nc);
            for (int i = 0; i < nc; ++i) {
                Component& c = comps_[i];
                c.id = d_[seg + 6 + 3 * i];
                c.h = d_[seg + 7 + 3 * i] >> 4;
                c.v = d_[seg + 7 + 3 * i] & 15;
                c.tq = d_[seg + 8 + 3 * i];
                if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) return fail("JPEG: unsupported sampling");
                hmax_ = std::max(hmax_, c.h);
                vmax_ = std::max(vmax_, c.v);
            }
            const int mcus_x = (width_ + 8 * hmax_ - 1) / (8 * hmax_), mcus_y = (height_ + 8 * vmax_ - 1) / (8 * vmax_);
            for (auto& c : comps_) {
                c.bw = mcus_x * c.h;
                c.bh = mcus_y * c.v;
                c.plane.assign((size_t)c.bw * 8 * c.bh * 8, 0);
            }
            frame = true;
        } else if (marker >= 0xC2 && marker <= 0xCF && marker != 0xC4 && marker != 0xC8 && marker != 0xCC) {
            return fail("JPEG: progressive, lossless or arithmetic-coded files are not supported");
        } else if (marker == 0xDD) {  // DRI
            if (len - 2 < 2) return fail("JPEG: truncated restart interval");
            restart_ = read_u16(seg);
        } else if (marker == 0xDA) {  // SOS
            if (!frame) return fail("JPEG: scan before frame header");
            if (len - 2 < 1) return fail("JPEG: truncated scan header");
            const int ns = d_[seg];
            if (1 + 2 * ns > len - 2) return fail("JPEG: truncated scan header");
            for (int i = 0; i < ns; ++i) {
                const int cid = d_[seg + 1 + 2 * i], t = d_[seg + 2 + 2 * i];
                const int td = t >> 4, ta = t & 15;
                if (td > 3 || ta > 3) return fail("JPEG: bad Huffman table selector");
                bool found = false;
                for (auto& c : comps_)
                    if (c.id == cid) { c.td = td; c.ta = ta; found = true; }
                if (!found) return fail("JPEG: scan names an unknown component");
            }
            if (ns != (int)comps_.size()) return fail("JPEG: non-interleaved multi-scan files are not supported");
            pos_ = seg + len - 2;
            if (decode_scan()) return -1;
            // continue after the entropy-coded segment
            while (pos_ + 1 < n_ && !(d_[pos_] == 0xFF && d_[pos_ + 1] != 0x00 &&
                                      !(d_[pos_ + 1] >= 0xD0 && d_[pos_ + 1] <= 0xD7)))
                ++pos_;
            continue;
        }
        pos_ = seg + len - 2;
    }
    if (!frame) return fail("JPEG: no frame");
    W = width_;
    H = height_;
    bgr.resize((size_t)W * H * 3);
    // chroma upsampling by the triangle filter (3/4 nearer sample, 1/4 farther), then YCbCr -> RGB
    auto sample = [&](const Component& c, int x, int y) -> double {
        const int pw = c.bw * 8, ph = c.bh * 8;
        if (c.h == hmax_ && c.v == vmax_) return c.plane[(size_t)y * pw + x];
        const int rx = hmax_ / c.h, ry = vmax_ / c.v;
        if (rx > 2 || ry > 2 || hmax_ % c.h || vmax_ % c.v)  // other ratios: replication, as libjpeg does
            return c.plane[(size_t)(y * c.v / vmax_) * pw + (x * c.h / hmax_)];
        // position in the component plane of the full-resolution sample centre
        const double fx = (x + 0.5) * c.h / hmax_ - 0.5, fy = (y + 0.5) * c.v / vmax_ - 0.5;
        const int x0 = (int)std::floor(fx), y0 = (int)std::floor(fy);
        const double ax = fx - x0, ay = fy - y0;
        const int cw = (width_ * c.h + hmax_ - 1) / hmax_, chh = (height_ * c.v + vmax_ - 1) / vmax_;
        auto at = [&](int xx, int yy) -> double {
            xx = xx < 0 ? 0 : (xx >= cw ? cw - 1 : xx);
            yy = yy < 0 ? 0 : (yy >= chh ? chh - 1 : yy);
            (void)ph;
            return c.plane[(size_t)yy * pw + xx];
        };
        return (1 - ay) * ((1 - ax) * at(x0, y0) + ax * at(x0 + 1, y0)) + ay * ((1 - ax) * at(x0, y0 + 1) + ax * at(x0 + 1, y0 + 1));
    };
    auto clamp8 = [](double v) -> uint8_t {
        const long r = std::lround(v);
        return (uint8_t)(r < 0 ? 0 : (r > 255 ? 255 : r));
    };
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            uint8_t* o = bgr.data() + ((size_t)y * W + x) * 3;
            if (comps_.size() == 1) {
                o[0] = o[1] = o[2] = comps_[0].plane[(size_t)y * comps_[0].bw * 8 + x];
                continue;
            }
            const double Y = sample(comps_[0], x, y), cb = sample(comps_[1], x, y) - 128.0,
                         cr = sample(comps_[2], x, y) - 128.0;
            o[2] = clamp8(Y + 1.402 * cr);
            o[1] = clamp8(Y - 0.344136 * cb - 0.714136 * cr);
            o[0] = clamp8(Y + 1.772 * cb);
        }
    return 0;
}

}  // namespace

extern "C" {

int hpm_decode_image(const uint8_t* bytes, size_t n, uint8_t** bgr, int* w, int* h) {
    if (!bytes || !bgr || !w || !h) return fail("hpm_decode_image: null argument");
    *bgr = nullptr;
    std::vector<uint8_t> out;
    int W = 0, H = 0, rc;
    static const uint8_t png_sig[8] = { 0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A };
    if (n >= 8 && !std::memcmp(bytes, png_sig, 8)) rc = decode_png(bytes, n, out, W, H);
    else if (n >= 4 && bytes[0] == 0xFF && bytes[1] == 0xD8) rc = Jpeg(bytes, n).decode(out, W, H);
    else rc = fail("unknown image format (PNG and baseline JPEG are read)");
    if (rc) return rc;
    *bgr = static_cast<uint8_t*>(std::malloc(out.size()));
    if (!*bgr) return fail("out of memory");
    std::memcpy(*bgr, out.data(), out.size());
    *w = W;
    *h = H;
    return 0;
}

void hpm_free_image(uint8_t* bgr) { std::free(bgr); }

const char* hpm_image_error(void) { return g_error.c_str(); }

}  // extern "C"
