// Minimal .npy reader/writer exposing the small subset of the third-party
// `cnpy` API (rogersce/cnpy, no pinned version; linked from /usr/local by
// src/Makefile:14,23 of the reference) that the reference's two programs call:
//   cnpy::NpyArray{shape, data<T>()}            src/build_model.cu:1004-1019
//   cnpy::npy_load(std::string)                 src/spvi_2.cu:368
//   cnpy::npy_save(fname, const T*, shape, mode) src/build_model.cu:1305-1310,
//                                                src/spvi_2.cu:790-791
// cnpy is not installed in this image and there is no network, so this header
// is written from the public NumPy .npy format description (magic, version,
// little-endian header length, Python-dict header, C-order payload).  It does
// I/O only; no arithmetic of the reference passes through it.
//
// Test infrastructure: used only to compile the reference into oracle/_ref.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <typeinfo>
#include <vector>

namespace cnpy {

struct NpyArray {
  std::vector<size_t> shape;
  size_t word_size = 0;
  bool fortran_order = false;
  size_t num_vals = 0;
  std::shared_ptr<std::vector<char>> bytes;

  template <typename T> T* data() { return reinterpret_cast<T*>(bytes->data()); }
  template <typename T> const T* data() const {
    return reinterpret_cast<const T*>(bytes->data());
  }
  size_t num_bytes() const { return bytes ? bytes->size() : 0; }
};

namespace detail {

inline std::string parse_field(const std::string& hdr, const std::string& key) {
  size_t k = hdr.find("'" + key + "'");
  if (k == std::string::npos) throw std::runtime_error("npy header: missing " + key);
  size_t c = hdr.find(':', k);
  return hdr.substr(c + 1);
}

inline void parse_header(const std::string& hdr, size_t& word_size,
                         std::vector<size_t>& shape, bool& fortran) {
  std::string d = parse_field(hdr, "descr");
  size_t q0 = d.find('\'');
  size_t q1 = d.find('\'', q0 + 1);
  std::string descr = d.substr(q0 + 1, q1 - q0 - 1);
  // descr like '<f4', '<i8', '|u1'
  size_t digits = descr.find_first_of("0123456789");
  word_size = std::stoul(descr.substr(digits));
  std::string f = parse_field(hdr, "fortran_order");
  fortran = f.find("True") < f.find(',');
  std::string s = parse_field(hdr, "shape");
  size_t p0 = s.find('(');
  size_t p1 = s.find(')');
  std::string inner = s.substr(p0 + 1, p1 - p0 - 1);
  shape.clear();
  size_t pos = 0;
  while (pos < inner.size()) {
    size_t comma = inner.find(',', pos);
    std::string tok = inner.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
    size_t a = tok.find_first_of("0123456789");
    if (a != std::string::npos) shape.push_back(std::stoull(tok.substr(a)));
    if (comma == std::string::npos) break;
    pos = comma + 1;
  }
}

template <typename T> char type_char() {
  if (typeid(T) == typeid(float) || typeid(T) == typeid(double)) return 'f';
  if (typeid(T) == typeid(int8_t) || typeid(T) == typeid(int16_t) ||
      typeid(T) == typeid(int32_t) || typeid(T) == typeid(int64_t) ||
      typeid(T) == typeid(long) || typeid(T) == typeid(long long) || typeid(T) == typeid(char))
    return 'i';
  if (typeid(T) == typeid(bool)) return 'b';
  return 'u';
}

}  // namespace detail

inline NpyArray npy_load(const std::string& fname) {
  FILE* fp = std::fopen(fname.c_str(), "rb");
  if (!fp) throw std::runtime_error("npy_load: cannot open " + fname);
  char magic[8];
  if (std::fread(magic, 1, 8, fp) != 8 || std::memcmp(magic, "\x93NUMPY", 6) != 0) {
    std::fclose(fp);
    throw std::runtime_error("npy_load: bad magic in " + fname);
  }
  uint32_t hlen = 0;
  if (magic[6] == 1) {
    uint16_t h16;
    if (std::fread(&h16, 2, 1, fp) != 1) { std::fclose(fp); throw std::runtime_error("npy_load: short"); }
    hlen = h16;
  } else {
    if (std::fread(&hlen, 4, 1, fp) != 1) { std::fclose(fp); throw std::runtime_error("npy_load: short"); }
  }
  std::string hdr(hlen, '\0');
  if (std::fread(&hdr[0], 1, hlen, fp) != hlen) { std::fclose(fp); throw std::runtime_error("npy_load: short"); }
  NpyArray arr;
  detail::parse_header(hdr, arr.word_size, arr.shape, arr.fortran_order);
  arr.num_vals = 1;
  for (size_t d : arr.shape) arr.num_vals *= d;
  arr.bytes = std::make_shared<std::vector<char>>(arr.num_vals * arr.word_size);
  size_t got = std::fread(arr.bytes->data(), 1, arr.bytes->size(), fp);
  std::fclose(fp);
  if (got != arr.bytes->size()) throw std::runtime_error("npy_load: truncated " + fname);
  return arr;
}

template <typename T>
void npy_save(std::string fname, const T* data, const std::vector<size_t> shape,
              std::string mode = "w") {
  if (mode != "w") throw std::runtime_error("npy_save: only mode \"w\" is supported");
  std::string dict = "{'descr': '<";
  dict += detail::type_char<T>();
  dict += std::to_string(sizeof(T));
  dict += "', 'fortran_order': False, 'shape': (";
  for (size_t i = 0; i < shape.size(); ++i) {
    dict += std::to_string(shape[i]);
    if (shape.size() == 1 || i + 1 < shape.size()) dict += ",";
    if (i + 1 < shape.size()) dict += " ";
  }
  dict += "), }";
  // pad so that magic(6)+ver(2)+len(2)+dict+'\n' is a multiple of 64
  size_t total = 10 + dict.size() + 1;
  size_t pad = (64 - total % 64) % 64;
  dict.append(pad, ' ');
  dict += '\n';
  FILE* fp = std::fopen(fname.c_str(), "wb");
  if (!fp) throw std::runtime_error("npy_save: cannot open " + fname);
  const char magic[8] = {'\x93', 'N', 'U', 'M', 'P', 'Y', 1, 0};
  std::fwrite(magic, 1, 8, fp);
  uint16_t hl = (uint16_t)dict.size();
  std::fwrite(&hl, 2, 1, fp);
  std::fwrite(dict.data(), 1, dict.size(), fp);
  size_t n = 1;
  for (size_t d : shape) n *= d;
  if (n) std::fwrite(data, sizeof(T), n, fp);
  std::fclose(fp);
}

}  // namespace cnpy
