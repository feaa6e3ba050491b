// npz_writer.cpp — see npz_writer.h.  Format: NPY 1.0 headers (magic, version,
// little-endian header length, Python-literal dict padded to 64 bytes) inside
// a zip archive with stored (method 0) entries and CRC-32 checksums.
#include "npz_writer.h"

#include <cstdio>
#include <cstring>

namespace cupf_host {

static uint32_t crc32(const std::string& s) {
  static uint32_t table[256];
  static bool init = false;
  if (!init) {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      table[i] = c;
    }
    init = true;
  }
  uint32_t c = 0xFFFFFFFFu;
  for (unsigned char b : s) c = table[(c ^ b) & 0xFF] ^ (c >> 8);
  return c ^ 0xFFFFFFFFu;
}

void NpzWriter::add_raw(const std::string& name, const char* descr, const void* data,
                        size_t count, size_t elem) {
  std::string hdr = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (" +
                    std::to_string(count) + ",), }";
  const size_t pre = 10;  // magic(6) + version(2) + header length(2)
  size_t total = pre + hdr.size() + 1;
  const size_t pad = (64 - total % 64) % 64;
  hdr.append(pad, ' ');
  hdr.push_back('\n');
  std::string b;
  b.append("\x93NUMPY", 6);
  b.push_back('\x01');
  b.push_back('\x00');
  const uint16_t hl = (uint16_t)hdr.size();
  b.push_back((char)(hl & 0xFF));
  b.push_back((char)(hl >> 8));
  b += hdr;
  b.append(static_cast<const char*>(data), count * elem);
  mEntries.push_back({name + ".npy", std::move(b)});
}

void NpzWriter::add(const std::string& name, const std::vector<float>& v) {
  add_raw(name, "<f4", v.data(), v.size(), 4);
}

void NpzWriter::add(const std::string& name, const std::vector<int>& v) {
  add_raw(name, "<i4", v.data(), v.size(), 4);
}

static void put16(std::string& s, uint16_t v) {
  s.push_back((char)(v & 0xFF));
  s.push_back((char)(v >> 8));
}
static void put32(std::string& s, uint32_t v) {
  for (int i = 0; i < 4; ++i) s.push_back((char)((v >> (8 * i)) & 0xFF));
}

bool NpzWriter::write(const std::string& path) const {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  std::string central;
  uint32_t offset = 0;
  bool ok = true;
  for (const Entry& e : mEntries) {
    const uint32_t crc = crc32(e.bytes);
    const uint32_t sz = (uint32_t)e.bytes.size();
    std::string h;
    put32(h, 0x04034b50u);
    put16(h, 20);
    put16(h, 0);
    put16(h, 0);  // stored
    put16(h, 0);
    put16(h, 0x21);  // 1980-01-01
    put32(h, crc);
    put32(h, sz);
    put32(h, sz);
    put16(h, (uint16_t)e.name.size());
    put16(h, 0);
    h += e.name;
    ok = ok && std::fwrite(h.data(), 1, h.size(), f) == h.size();
    ok = ok && std::fwrite(e.bytes.data(), 1, e.bytes.size(), f) == e.bytes.size();
    std::string c;
    put32(c, 0x02014b50u);
    put16(c, 20);
    put16(c, 20);
    put16(c, 0);
    put16(c, 0);
    put16(c, 0);
    put16(c, 0x21);
    put32(c, crc);
    put32(c, sz);
    put32(c, sz);
    put16(c, (uint16_t)e.name.size());
    put16(c, 0);
    put16(c, 0);
    put16(c, 0);
    put16(c, 0);
    put32(c, 0);
    put32(c, offset);
    c += e.name;
    central += c;
    offset += (uint32_t)(h.size() + e.bytes.size());
  }
  std::string end;
  put32(end, 0x06054b50u);
  put16(end, 0);
  put16(end, 0);
  put16(end, (uint16_t)mEntries.size());
  put16(end, (uint16_t)mEntries.size());
  put32(end, (uint32_t)central.size());
  put32(end, offset);
  put16(end, 0);
  ok = ok && std::fwrite(central.data(), 1, central.size(), f) == central.size();
  ok = ok && std::fwrite(end.data(), 1, end.size(), f) == end.size();
  return std::fclose(f) == 0 && ok;
}

}  // namespace cupf_host
