// Run-time reader of the reference's configuration header.
//
// The reference compiles its problem into the builder: src/build_model.cu:932
// includes input_to_build_model.h inside main, a list of C declarations such as
//   int32_t nt = 50;  float dx = 1; float dy = dx;  int32_t i_term = (int)(0.5*gsize);
// The drop-in build_model reads the same file at run time instead, so a user
// keeps editing the header as before without recompiling.  Supported: the
// declaration types std::string / float / double / int / int32_t, numeric
// literals, previously declared names, + - * /, parentheses and (int)/(float)
// casts, with C's integer division for integer operands.
#pragma once

#include <cctype>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>

namespace e2e {
namespace cfg {

struct Val {
  double v = 0;
  bool is_int = false;
  std::string s;
  bool is_str = false;
};

class Header {
 public:
  std::map<std::string, Val> vars;

  void parse(const std::string& text) {
    std::string t = strip_comments(text);
    size_t pos = 0;
    while (true) {
      size_t semi = t.find(';', pos);
      if (semi == std::string::npos) break;
      statement(t.substr(pos, semi - pos));
      pos = semi + 1;
    }
  }
  void parse_file(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    parse(ss.str());
  }
  bool has(const std::string& k) const { return vars.count(k) != 0; }
  double num(const std::string& k) const {
    auto it = vars.find(k);
    if (it == vars.end()) throw std::runtime_error("config header lacks " + k);
    return it->second.v;
  }
  std::string str(const std::string& k) const {
    auto it = vars.find(k);
    if (it == vars.end() || !it->second.is_str) throw std::runtime_error("config header lacks string " + k);
    return it->second.s;
  }

 private:
  const char* p_ = nullptr;

  static std::string strip_comments(const std::string& in) {
    std::string o;
    for (size_t i = 0; i < in.size(); ++i) {
      if (in[i] == '/' && i + 1 < in.size() && in[i + 1] == '/') {
        while (i < in.size() && in[i] != '\n') ++i;
        o += '\n';
      } else if (in[i] == '/' && i + 1 < in.size() && in[i + 1] == '*') {
        i += 2;
        while (i + 1 < in.size() && !(in[i] == '*' && in[i + 1] == '/')) ++i;
        ++i;
      } else if (in[i] == '"') {
        o += in[i++];
        while (i < in.size() && in[i] != '"') o += in[i++];
        if (i < in.size()) o += in[i];
      } else {
        o += in[i];
      }
    }
    return o;
  }

  static std::string trim(const std::string& s) {
    size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
    return a == std::string::npos ? "" : s.substr(a, b - a + 1);
  }

  void statement(const std::string& raw) {
    std::string s = trim(raw);
    if (s.empty() || s[0] == '#') return;
    size_t eq = s.find('=');
    if (eq == std::string::npos) return;  // declaration without initialiser: ignore
    std::string lhs = trim(s.substr(0, eq)), rhs = trim(s.substr(eq + 1));
    size_t sp = lhs.find_last_of(" \t*&");
    std::string type = trim(lhs.substr(0, sp == std::string::npos ? 0 : sp));
    std::string name = trim(lhs.substr(sp == std::string::npos ? 0 : sp + 1));
    if (type.rfind("extern", 0) == 0) return;
    Val v;
    if (type.find("string") != std::string::npos) {
      size_t q0 = rhs.find('"'), q1 = rhs.rfind('"');
      if (q0 == std::string::npos || q1 == q0) throw std::runtime_error("bad string for " + name);
      v.is_str = true;
      v.s = rhs.substr(q0 + 1, q1 - q0 - 1);
    } else {
      p_ = rhs.c_str();
      v = expr();
      skip();
      if (*p_) throw std::runtime_error("cannot parse initialiser of " + name + ": " + rhs);
      if (type.find("int") != std::string::npos || type == "long" || type == "long long") {
        v.v = std::trunc(v.v);
        v.is_int = true;
      } else if (type == "float") {
        v.v = (double)(float)v.v;
        v.is_int = false;
      } else {
        v.is_int = false;
      }
    }
    vars[name] = v;
  }

  void skip() {
    while (*p_ && std::isspace((unsigned char)*p_)) ++p_;
  }

  Val expr() {
    Val a = term();
    while (true) {
      skip();
      char c = *p_;
      if (c != '+' && c != '-') return a;
      ++p_;
      Val b = term();
      a = arith(a, b, c);
    }
  }
  Val term() {
    Val a = unary();
    while (true) {
      skip();
      char c = *p_;
      if (c != '*' && c != '/') return a;
      ++p_;
      Val b = unary();
      a = arith(a, b, c);
    }
  }
  static Val arith(const Val& a, const Val& b, char op) {
    Val r;
    r.is_int = a.is_int && b.is_int;
    switch (op) {
      case '+': r.v = a.v + b.v; break;
      case '-': r.v = a.v - b.v; break;
      case '*': r.v = a.v * b.v; break;
      case '/':
        if (b.v == 0) throw std::runtime_error("division by zero in config header");
        r.v = r.is_int ? std::trunc(a.v / b.v) : a.v / b.v;
        break;
    }
    return r;
  }
  Val unary() {
    skip();
    if (*p_ == '-') {
      ++p_;
      Val v = unary();
      v.v = -v.v;
      return v;
    }
    if (*p_ == '+') {
      ++p_;
      return unary();
    }
    return primary();
  }
  Val primary() {
    skip();
    if (*p_ == '(') {
      const char* save = p_;
      ++p_;
      skip();
      std::string ident;
      while (std::isalnum((unsigned char)*p_) || *p_ == '_') ident += *p_++;
      skip();
      if (*p_ == ')' && (ident == "int" || ident == "int32_t" || ident == "float" || ident == "double" || ident == "long")) {
        ++p_;
        Val v = unary();
        if (ident == "float") {
          v.v = (double)(float)v.v;
          v.is_int = false;
        } else if (ident == "double") {
          v.is_int = false;
        } else {
          v.v = std::trunc(v.v);
          v.is_int = true;
        }
        return v;
      }
      p_ = save + 1;
      Val v = expr();
      skip();
      if (*p_ != ')') throw std::runtime_error("missing ')' in config header");
      ++p_;
      return v;
    }
    if (std::isdigit((unsigned char)*p_) || *p_ == '.') {
      char* end = nullptr;
      double d = std::strtod(p_, &end);
      std::string tok(p_, (const char*)end);
      p_ = end;
      Val v;
      v.v = d;
      v.is_int = tok.find_first_of(".eE") == std::string::npos;
      while (*p_ == 'f' || *p_ == 'F' || *p_ == 'l' || *p_ == 'L' || *p_ == 'u' || *p_ == 'U') {
        if (*p_ == 'f' || *p_ == 'F') v.is_int = false;
        ++p_;
      }
      return v;
    }
    std::string ident;
    while (std::isalnum((unsigned char)*p_) || *p_ == '_') ident += *p_++;
    if (ident.empty()) throw std::runtime_error("unexpected character in config header");
    auto it = vars.find(ident);
    if (it == vars.end()) throw std::runtime_error("unknown name in config header: " + ident);
    return it->second;
  }
};

}  // namespace cfg
}  // namespace e2e
