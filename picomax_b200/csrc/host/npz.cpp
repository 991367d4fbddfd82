// Reusable output: float64 arrays in a NumPy .npz container.
//
// The reference plans HDF5 output of its spectra for re-use by the wrappers
// (src/pmx_io.cpp:744-807: ReXij / ImXij datasets, commented out, README
// "HDF5 output support"); no HDF5 library is available to this build
// environment, so the same arrays go to the self-describing NumPy format
// instead, which numpy.load reads directly (and MATLAB through npy readers).
//
// Format (written from the published specifications):
//  * NPY 1.0: magic "\x93NUMPY", version 1.0, a little-endian uint16 header
//    length, an ASCII dict {'descr': '<f8', 'fortran_order': False,
//    'shape': (...), } padded with spaces and a final newline to a multiple
//    of 64 bytes, then the data in C order.
//  * ZIP (PKWARE APPNOTE): one "stored" (uncompressed) entry per array,
//    name "<array>.npy", each with a local file header, then the central
//    directory and the end-of-central-directory record. CRC-32 with the
//    reflected IEEE 802.3 polynomial 0xEDB88320. Sizes and offsets must fit
//    32 bits (no ZIP64): larger files are refused.
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../../include/picomax.h"

namespace {

uint32_t crc_table_entry(uint32_t c) {
  for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
  return c;
}

struct Crc32 {
  uint32_t table[256];
  Crc32() {
    for (uint32_t i = 0; i < 256; ++i) table[i] = crc_table_entry(i);
  }
  uint32_t update(uint32_t crc, const unsigned char* p, size_t n) const {
    crc = ~crc;
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return ~crc;
  }
};

void put16(std::string& s, uint32_t v) {
  s.push_back((char)(v & 0xFF));
  s.push_back((char)((v >> 8) & 0xFF));
}
void put32(std::string& s, uint32_t v) {
  put16(s, v & 0xFFFF);
  put16(s, v >> 16);
}

// NPY 1.0 header of a float64 C-order array
std::string npy_header(int ndim, const long long* shape) {
  std::string dict = "{'descr': '<f8', 'fortran_order': False, 'shape': (";
  for (int d = 0; d < ndim; ++d) dict += std::to_string(shape[d]) + ", ";
  dict += "), }";
  const size_t pre = 10;  // magic (6) + version (2) + header length (2)
  size_t total = pre + dict.size() + 1;
  total = (total + 63) / 64 * 64;
  dict.append(total - pre - dict.size() - 1, ' ');
  dict.push_back('\n');
  std::string h("\x93NUMPY", 6);
  h.push_back((char)1);
  h.push_back((char)0);
  put16(h, (uint32_t)dict.size());
  return h + dict;
}

struct Entry {
  std::string name;
  uint32_t crc, size, offset;
};

std::string local_header(const Entry& e) {
  std::string s;
  put32(s, 0x04034b50u);
  put16(s, 20);  // version needed: 2.0
  put16(s, 0);   // flags
  put16(s, 0);   // stored
  put16(s, 0);   // time
  put16(s, 0x21);  // date 1980-01-01
  put32(s, e.crc);
  put32(s, e.size);
  put32(s, e.size);
  put16(s, (uint32_t)e.name.size());
  put16(s, 0);
  return s + e.name;
}

std::string central_header(const Entry& e) {
  std::string s;
  put32(s, 0x02014b50u);
  put16(s, 20);  // made by
  put16(s, 20);  // needed
  put16(s, 0);
  put16(s, 0);
  put16(s, 0);
  put16(s, 0x21);
  put32(s, e.crc);
  put32(s, e.size);
  put32(s, e.size);
  put16(s, (uint32_t)e.name.size());
  put16(s, 0);  // extra
  put16(s, 0);  // comment
  put16(s, 0);  // disk
  put16(s, 0);  // internal attributes
  put32(s, 0);  // external attributes
  put32(s, e.offset);
  return s + e.name;
}

}  // namespace

extern "C" int pmx_write_npz(const char* path, int count, const char* const* names, const double* const* data,
                             const int* ndims, const long long* shapes) {
  if (!path || count < 0 || count > 0xFFFF || (count > 0 && (!names || !data || !ndims || !shapes)))
    return PMX_ERR_INVALID;
  static const Crc32 crc;
  std::vector<Entry> entries;
  std::vector<std::string> headers;
  std::vector<size_t> bytes;
  uint64_t off = 0;
  const long long* sh = shapes;
  for (int i = 0; i < count; ++i) {
    if (!names[i] || !names[i][0] || ndims[i] < 0 || ndims[i] > 32) return PMX_ERR_INVALID;
    long long n = 1;
    for (int d = 0; d < ndims[i]; ++d) {
      if (sh[d] < 0) return PMX_ERR_INVALID;
      n *= sh[d];
    }
    if (n > 0 && !data[i]) return PMX_ERR_INVALID;
    headers.push_back(npy_header(ndims[i], sh));
    sh += ndims[i];
    const uint64_t nb = (uint64_t)n * sizeof(double);
    const uint64_t size = headers.back().size() + nb;
    Entry e{std::string(names[i]) + ".npy", 0, (uint32_t)size, (uint32_t)off};
    if (size > 0xFFFFFFFFull || off > 0xFFFFFFFFull) return PMX_ERR_LIMIT;
    uint32_t c = crc.update(0, reinterpret_cast<const unsigned char*>(headers.back().data()), headers.back().size());
    c = crc.update(c, reinterpret_cast<const unsigned char*>(data[i]), (size_t)nb);
    e.crc = c;
    off += 30 + e.name.size() + size;
    entries.push_back(e);
    bytes.push_back((size_t)nb);
  }
  if (off > 0xFFFFFFFFull) return PMX_ERR_LIMIT;
  FILE* f = std::fopen(path, "wb");
  if (!f) return PMX_ERR_IO;
  bool ok = true;
  for (int i = 0; i < count && ok; ++i) {
    const std::string lh = local_header(entries[i]);
    ok = std::fwrite(lh.data(), 1, lh.size(), f) == lh.size() &&
         std::fwrite(headers[i].data(), 1, headers[i].size(), f) == headers[i].size() &&
         (bytes[i] == 0 || std::fwrite(data[i], 1, bytes[i], f) == bytes[i]);
  }
  std::string cd;
  for (const Entry& e : entries) cd += central_header(e);
  std::string end;
  put32(end, 0x06054b50u);
  put16(end, 0);
  put16(end, 0);
  put16(end, (uint32_t)count);
  put16(end, (uint32_t)count);
  put32(end, (uint32_t)cd.size());
  put32(end, (uint32_t)off);
  put16(end, 0);
  ok = ok && std::fwrite(cd.data(), 1, cd.size(), f) == cd.size() && std::fwrite(end.data(), 1, end.size(), f) == end.size();
  ok = (std::fclose(f) == 0) && ok;
  return ok ? PMX_OK : PMX_ERR_IO;
}
