// .npy reader/writer for the model and field files (NumPy format 1.0/2.0:
// magic "\x93NUMPY", version, little-endian header length, Python-literal
// dict {'descr', 'fortran_order', 'shape'}, then the C-order payload).
// The reference reads and writes these files through the third-party cnpy
// library (src/build_model.cu:1318-1349, :1305-1310; src/spvi_2.cu:360-410);
// this is an independent implementation of the same file format.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace e2e {
namespace npy {

struct Array {
  std::string descr;            // e.g. "<f4", "<i8", "<u4"
  std::vector<size_t> shape;
  std::vector<char> data;
  size_t count() const {
    size_t n = 1;
    for (size_t d : shape) n *= d;
    return n;
  }
  size_t word() const {
    size_t p = descr.find_first_of("0123456789");
    return p == std::string::npos ? 0 : (size_t)std::stoul(descr.substr(p));
  }
  char kind() const { return descr.size() >= 2 ? descr[1] : '?'; }
  template <typename T> const T* as() const { return reinterpret_cast<const T*>(data.data()); }
};

inline bool parse_header(const std::string& h, Array& a, bool& fortran, std::string& err) {
  size_t k = h.find("'descr'");
  if (k == std::string::npos) { err = "no descr"; return false; }
  size_t q0 = h.find('\'', h.find(':', k) + 1);
  size_t q1 = h.find('\'', q0 + 1);
  if (q0 == std::string::npos || q1 == std::string::npos) { err = "bad descr"; return false; }
  a.descr = h.substr(q0 + 1, q1 - q0 - 1);
  if (a.descr.size() >= 1 && a.descr[0] == '|') a.descr[0] = '<';
  if (a.descr.size() >= 1 && a.descr[0] == '>') { err = "big-endian arrays are not supported"; return false; }
  size_t f = h.find("'fortran_order'");
  fortran = false;
  if (f != std::string::npos) {
    size_t c = h.find(':', f);
    size_t t = h.find("True", c);
    size_t comma = h.find(',', c);
    fortran = (t != std::string::npos && (comma == std::string::npos || t < comma));
  }
  size_t s = h.find("'shape'");
  if (s == std::string::npos) { err = "no shape"; return false; }
  size_t p0 = h.find('(', s), p1 = h.find(')', p0);
  if (p0 == std::string::npos || p1 == std::string::npos) { err = "bad shape"; return false; }
  std::string in = h.substr(p0 + 1, p1 - p0 - 1);
  a.shape.clear();
  size_t pos = 0;
  while (pos < in.size()) {
    size_t c = in.find(',', pos);
    std::string tok = in.substr(pos, c == std::string::npos ? std::string::npos : c - pos);
    size_t d = tok.find_first_of("0123456789");
    if (d != std::string::npos) a.shape.push_back((size_t)std::stoull(tok.substr(d)));
    if (c == std::string::npos) break;
    pos = c + 1;
  }
  return true;
}

inline bool read(const std::string& path, Array& a, std::string& err) {
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) { err = "cannot open " + path; return false; }
  unsigned char mg[8];
  if (std::fread(mg, 1, 8, fp) != 8 || std::memcmp(mg, "\x93NUMPY", 6) != 0) {
    std::fclose(fp);
    err = "not an npy file: " + path;
    return false;
  }
  uint32_t hl = 0;
  if (mg[6] == 1) {
    uint16_t h16 = 0;
    if (std::fread(&h16, 2, 1, fp) != 1) { std::fclose(fp); err = "truncated " + path; return false; }
    hl = h16;
  } else {
    if (std::fread(&hl, 4, 1, fp) != 1) { std::fclose(fp); err = "truncated " + path; return false; }
  }
  std::string h(hl, '\0');
  if (hl && std::fread(&h[0], 1, hl, fp) != hl) { std::fclose(fp); err = "truncated " + path; return false; }
  bool fortran = false;
  if (!parse_header(h, a, fortran, err)) { std::fclose(fp); err += " in " + path; return false; }
  if (fortran && a.shape.size() > 1) {
    size_t nontriv = 0;
    for (size_t d : a.shape) nontriv += d > 1;
    if (nontriv > 1) { std::fclose(fp); err = "fortran-order arrays are not supported: " + path; return false; }
  }
  size_t bytes = a.count() * a.word();
  a.data.resize(bytes);
  size_t got = bytes ? std::fread(a.data.data(), 1, bytes, fp) : 0;
  std::fclose(fp);
  if (got != bytes) { err = "truncated payload in " + path; return false; }
  return true;
}

inline bool write(const std::string& path, const char* descr, const std::vector<size_t>& shape,
                  const void* data, std::string& err) {
  std::string d = std::string("{'descr': '") + descr + "', 'fortran_order': False, 'shape': (";
  for (size_t i = 0; i < shape.size(); ++i) {
    d += std::to_string(shape[i]);
    if (shape.size() == 1 || i + 1 < shape.size()) d += ",";
    if (i + 1 < shape.size()) d += " ";
  }
  d += "), }";
  size_t total = 10 + d.size() + 1;
  d.append((64 - total % 64) % 64, ' ');
  d += '\n';
  FILE* fp = std::fopen(path.c_str(), "wb");
  if (!fp) { err = "cannot create " + path; return false; }
  const unsigned char mg[8] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0};
  uint16_t hl = (uint16_t)d.size();
  bool ok = std::fwrite(mg, 1, 8, fp) == 8 && std::fwrite(&hl, 2, 1, fp) == 1 &&
            std::fwrite(d.data(), 1, d.size(), fp) == d.size();
  size_t n = 1;
  for (size_t s : shape) n *= s;
  size_t w = 0;
  {
    std::string ds(descr);
    size_t p = ds.find_first_of("0123456789");
    w = (size_t)std::stoul(ds.substr(p));
  }
  if (ok && n) ok = std::fwrite(data, w, n, fp) == n;
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok) err = "write failed: " + path;
  return ok;
}

}  // namespace npy
}  // namespace e2e
