// fa2_png.cpp -- a small PNG writer for the rendered layouts: 8-bit RGB,
// scanlines with filter 0, the zlib stream made of stored (uncompressed)
// deflate blocks, CRC-32 and Adler-32 computed here.  The reference writes
// PNGs through pngwriter and libpng, neither of which is present; this
// encoder follows the PNG format itself (signature, IHDR, IDAT, IEND).
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <vector>

#include "fa2b200.h"

namespace {

uint32_t crc_table[256];
bool crc_ready = false;

void crc_init() {
    for (uint32_t n = 0; n < 256; ++n) {
        uint32_t c = n;
        for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
        crc_table[n] = c;
    }
    crc_ready = true;
}

uint32_t crc32_of(const uint8_t *p, size_t n, uint32_t c = 0xffffffffu) {
    if (!crc_ready) crc_init();
    for (size_t i = 0; i < n; ++i) c = crc_table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}

void put32(std::vector<uint8_t> &o, uint32_t v) {
    o.push_back((uint8_t)(v >> 24));
    o.push_back((uint8_t)(v >> 16));
    o.push_back((uint8_t)(v >> 8));
    o.push_back((uint8_t)v);
}

void chunk(std::vector<uint8_t> &o, const char *type, const std::vector<uint8_t> &data) {
    put32(o, (uint32_t)data.size());
    const size_t at = o.size();
    o.insert(o.end(), type, type + 4);
    o.insert(o.end(), data.begin(), data.end());
    put32(o, crc32_of(o.data() + at, o.size() - at) ^ 0xffffffffu);
}

}  // namespace

extern "C" int fa2_png_encode(const uint8_t *rgb, int32_t w, int32_t h, const char *path) {
    if (!rgb || w <= 0 || h <= 0 || !path) return FA2_ERR_INVALID_ARGUMENT;
    std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<uint8_t> ihdr;
    put32(ihdr, (uint32_t)w);
    put32(ihdr, (uint32_t)h);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(2);  // colour type: RGB
    ihdr.push_back(0);  // deflate
    ihdr.push_back(0);  // adaptive filtering (every line filter 0)
    ihdr.push_back(0);  // no interlace
    chunk(out, "IHDR", ihdr);
    // raw image: a filter byte then the row's RGB bytes, per row
    const size_t row = 3 * (size_t)w;
    std::vector<uint8_t> raw;
    raw.reserve((row + 1) * (size_t)h);
    for (int y = 0; y < h; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb + (size_t)y * row, rgb + (size_t)(y + 1) * row);
    }
    // zlib: header, stored blocks of at most 65535 bytes, Adler-32
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t pos = 0;
    do {
        const size_t len = std::min<size_t>(65535, raw.size() - pos);
        const bool last = pos + len == raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)len);
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len);
        z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + pos, raw.begin() + pos + len);
        pos += len;
    } while (pos < raw.size());
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) {
        a = (a + c) % 65521;
        b = (b + a) % 65521;
    }
    put32(z, (b << 16) | a);
    chunk(out, "IDAT", z);
    chunk(out, "IEND", {});
    FILE *f = fopen(path, "wb");
    if (!f) return FA2_ERR_IO;
    const bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
    return fclose(f) == 0 && ok ? FA2_OK : FA2_ERR_IO;
}
