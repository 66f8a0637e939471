#include "fm_image_io.h"

#include <zlib.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace fmhost {

namespace {

std::vector<uint8_t> read_file(const std::string& path)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open image: " + path);
    return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void rgbe_to_float(const uint8_t* e, float* out)
{
    if (e[3] != 0) {
        const float f = std::ldexp(1.0f, (int)e[3] - 136);
        out[0] = e[0] * f;
        out[1] = e[1] * f;
        out[2] = e[2] * f;
    } else {
        out[0] = out[1] = out[2] = 0.0f;
    }
}

ImageF read_hdr(const std::string& path)
{
    const std::vector<uint8_t> d = read_file(path);
    size_t p = 0;
    auto line = [&]() {
        std::string s;
        while (p < d.size() && d[p] != '\n') s += (char)d[p++];
        if (p < d.size()) ++p;
        return s;
    };
    const std::string magic = line();
    if (magic.rfind("#?RADIANCE", 0) != 0 && magic.rfind("#?RGBE", 0) != 0)
        throw std::runtime_error("not a Radiance file: " + path);
    for (;;) {
        if (p >= d.size()) throw std::runtime_error("truncated hdr header: " + path);
        const std::string l = line();
        if (l.empty()) break;
        if (l.rfind("FORMAT=", 0) == 0 && l != "FORMAT=32-bit_rle_rgbe")
            throw std::runtime_error("unsupported hdr format: " + path);
    }
    const std::string res = line();
    int h = 0, w = 0;
    if (std::sscanf(res.c_str(), "-Y %d +X %d", &h, &w) != 2 || w <= 0 || h <= 0)
        throw std::runtime_error("unsupported hdr orientation: " + path);
    ImageF img;
    img.width = w;
    img.height = h;
    img.rgb.assign((size_t)w * h * 3, 0.0f);
    std::vector<uint8_t> scan((size_t)w * 4);
    auto need = [&](size_t n) {
        if (p + n > d.size()) throw std::runtime_error("truncated hdr data: " + path);
    };
    for (int y = 0; y < h; ++y) {
        bool rle = false;
        if (w >= 8 && w < 32768) {
            need(4);
            rle = d[p] == 2 && d[p + 1] == 2 && !(d[p + 2] & 0x80);
        }
        if (!rle) {
            // flat scanlines from here to the end of the image
            const size_t remaining = (size_t)(h - y) * w * 4;
            need(remaining);
            for (size_t q = 0; q < (size_t)(h - y) * w; ++q)
                rgbe_to_float(&d[p + 4 * q], &img.rgb[((size_t)y * w) * 3 + 3 * q]);
            return img;
        }
        if (((int)d[p + 2] << 8 | d[p + 3]) != w) throw std::runtime_error("bad hdr scanline width: " + path);
        p += 4;
        for (int c = 0; c < 4; ++c) {
            int x = 0;
            while (x < w) {
                need(1);
                int count = d[p++];
                if (count > 128) {
                    count -= 128;
                    need(1);
                    const uint8_t v = d[p++];
                    if (x + count > w) throw std::runtime_error("bad hdr run: " + path);
                    for (int k = 0; k < count; ++k) scan[(size_t)4 * (x + k) + c] = v;
                } else {
                    if (count == 0 || x + count > w) throw std::runtime_error("bad hdr dump: " + path);
                    need((size_t)count);
                    for (int k = 0; k < count; ++k) scan[(size_t)4 * (x + k) + c] = d[p++];
                }
                x += count;
            }
        }
        for (int x = 0; x < w; ++x) rgbe_to_float(&scan[(size_t)4 * x], &img.rgb[((size_t)y * w + x) * 3]);
    }
    return img;
}

uint32_t be32(const uint8_t* q) { return (uint32_t)q[0] << 24 | (uint32_t)q[1] << 16 | (uint32_t)q[2] << 8 | q[3]; }

int paeth(int a, int b, int c)
{
    const int p = a + b - c;
    const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

ImageF read_png(const std::string& path)
{
    const std::vector<uint8_t> d = read_file(path);
    static const uint8_t sig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
    if (d.size() < 8 || std::memcmp(d.data(), sig, 8) != 0) throw std::runtime_error("not a PNG file: " + path);
    size_t p = 8;
    int w = 0, h = 0, depth = 0, ctype = 0, interlace = 0;
    std::vector<uint8_t> idat, palette;
    while (p + 8 <= d.size()) {
        const uint32_t len = be32(&d[p]);
        const std::string type(reinterpret_cast<const char*>(&d[p + 4]), 4);
        if (p + 12 + len > d.size()) throw std::runtime_error("truncated PNG: " + path);
        const uint8_t* c = &d[p + 8];
        if (type == "IHDR") {
            w = (int)be32(c);
            h = (int)be32(c + 4);
            depth = c[8];
            ctype = c[9];
            interlace = c[12];
        } else if (type == "PLTE") {
            palette.assign(c, c + len);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), c, c + len);
        } else if (type == "IEND") {
            break;
        }
        p += 12 + len;
    }
    if (w <= 0 || h <= 0 || depth != 8 || interlace != 0)
        throw std::runtime_error("unsupported PNG (8-bit, non-interlaced only): " + path);
    int ch;
    switch (ctype) {
    case 0: ch = 1; break;
    case 2: ch = 3; break;
    case 3: ch = 1; break;
    case 4: ch = 2; break;
    case 6: ch = 4; break;
    default: throw std::runtime_error("unsupported PNG colour type: " + path);
    }
    const size_t stride = (size_t)w * ch;
    std::vector<uint8_t> raw((stride + 1) * h);
    uLongf raw_len = (uLongf)raw.size();
    if (uncompress(raw.data(), &raw_len, idat.data(), (uLong)idat.size()) != Z_OK || raw_len != raw.size())
        throw std::runtime_error("PNG inflate failed: " + path);
    std::vector<uint8_t> px(stride * h), prev(stride, 0);
    for (int y = 0; y < h; ++y) {
        const uint8_t f = raw[y * (stride + 1)];
        const uint8_t* in = &raw[y * (stride + 1) + 1];
        uint8_t* out = &px[y * stride];
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= (size_t)ch ? out[x - ch] : 0;
            const int b = prev[x];
            const int cc = x >= (size_t)ch ? prev[x - ch] : 0;
            int v = in[x];
            switch (f) {
            case 0: break;
            case 1: v += a; break;
            case 2: v += b; break;
            case 3: v += (a + b) / 2; break;
            case 4: v += paeth(a, b, cc); break;
            default: throw std::runtime_error("bad PNG filter: " + path);
            }
            out[x] = (uint8_t)v;
        }
        std::memcpy(prev.data(), out, stride);
    }
    ImageF img;
    img.width = w;
    img.height = h;
    img.rgb.resize((size_t)w * h * 3);
    for (size_t q = 0; q < (size_t)w * h; ++q) {
        uint8_t rgb[3];
        const uint8_t* s = &px[q * ch];
        if (ctype == 3) {
            const size_t k = 3 * (size_t)s[0];
            if (k + 2 >= palette.size()) throw std::runtime_error("bad PNG palette index: " + path);
            rgb[0] = palette[k];
            rgb[1] = palette[k + 1];
            rgb[2] = palette[k + 2];
        } else if (ch <= 2) {
            rgb[0] = rgb[1] = rgb[2] = s[0];
        } else {
            rgb[0] = s[0];
            rgb[1] = s[1];
            rgb[2] = s[2];
        }
        for (int k = 0; k < 3; ++k) img.rgb[3 * q + k] = srgb_to_linear((float)rgb[k] / 255.0f);
    }
    return img;
}

void put32(std::string& s, uint32_t v)
{
    s += (char)(v >> 24);
    s += (char)(v >> 16);
    s += (char)(v >> 8);
    s += (char)v;
}

void chunk(std::string& out, const char* type, const std::string& data)
{
    put32(out, (uint32_t)data.size());
    std::string td = std::string(type, 4) + data;
    out += td;
    put32(out, (uint32_t)crc32(0L, reinterpret_cast<const Bytef*>(td.data()), (uInt)td.size()));
}

}  // namespace

float srgb_to_linear(float c)
{
    if (c <= 0.04045f) return c * 1.0f / 12.92f;
    return std::pow((c + 0.055f) * 1.0f / 1.055f, 2.4f);
}

float linear_to_srgb(float c)
{
    if (c <= 0.0031308f) return 12.92f * c;
    return 1.055f * std::pow(c, 1.0f / 2.4f) - 0.055f;
}

ImageF read_image(const std::string& path, bool is_hdr) { return is_hdr ? read_hdr(path) : read_png(path); }

void write_png(const std::string& path, int w, int h, const float* rgb)
{
    std::vector<uint8_t> q((size_t)3 * w * h);
    for (size_t i = 0; i < q.size(); ++i) {
        float c = rgb[i];
        c = c > 1.0f ? 1.0f : (c < 0.0f ? 0.0f : c);
        if (!(c == c)) c = 0.0f;
        q[i] = (uint8_t)std::lround(255.0f * c);
    }
    write_png_u8(path, w, h, q.data());
}

void write_png_u8(const std::string& path, int w, int h, const uint8_t* rgb8)
{
    std::string raw;
    raw.reserve((size_t)(3 * w + 1) * h);
    for (int y = 0; y < h; ++y) {
        raw += (char)0;
        raw.append(reinterpret_cast<const char*>(rgb8) + (size_t)y * 3 * w, (size_t)3 * w);
    }
    uLongf cap = compressBound((uLong)raw.size());
    std::string z(cap, '\0');
    if (compress2(reinterpret_cast<Bytef*>(&z[0]), &cap, reinterpret_cast<const Bytef*>(raw.data()), (uLong)raw.size(), 6) != Z_OK)
        throw std::runtime_error("PNG deflate failed");
    z.resize(cap);
    std::string out("\x89PNG\r\n\x1a\n", 8);
    std::string ihdr;
    put32(ihdr, (uint32_t)w);
    put32(ihdr, (uint32_t)h);
    ihdr += (char)8;
    ihdr += (char)2;
    ihdr += std::string(3, '\0');
    chunk(out, "IHDR", ihdr);
    chunk(out, "IDAT", z);
    chunk(out, "IEND", "");
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    f.write(out.data(), (std::streamsize)out.size());
}

void write_hdr(const std::string& path, int w, int h, const float* rgb)
{
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    std::ostringstream hdr;
    hdr << "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y " << h << " +X " << w << "\n";
    f << hdr.str();
    for (size_t q = 0; q < (size_t)w * h; ++q) {
        const float* c = rgb + 3 * q;
        const float m = std::fmax(c[0], std::fmax(c[1], c[2]));
        uint8_t e[4] = {0, 0, 0, 0};
        if (m >= 1e-32f) {
            int ex;
            const float norm = std::frexp(m, &ex) * 256.0f / m;
            e[0] = (uint8_t)(c[0] * norm);
            e[1] = (uint8_t)(c[1] * norm);
            e[2] = (uint8_t)(c[2] * norm);
            e[3] = (uint8_t)(ex + 128);
        }
        f.write(reinterpret_cast<const char*>(e), 4);
    }
}

}  // namespace fmhost
