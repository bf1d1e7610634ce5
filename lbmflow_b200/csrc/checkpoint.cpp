// Checkpoint/restart files in the reference's v3 format: writer, reader,
// hashes and the host-only C ABI entries (lbmb_checkpoint_write_host,
// lbmb_checkpoint_read_host, lbmb_fnv1a64).
//
// Reference: crates/lbm-core/src/solver.rs:29-44 (format constants),
// 84-118 (manifest, rank entry, section table, rank header), 831-1058
// (hashes, names, real codec), 1108-1215 (rank file reader), 1217-1287
// (scalar section), 4536-4724 (writer, manifest, save), 4739-5066 (restore).
#include "checkpoint.hpp"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>
#include <thread>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <sys/types.h>
#include <unistd.h>

#include "../../include/lbmb.h"

namespace lbmb {
extern thread_local std::string g_last_error;

namespace ckpt {
namespace {

constexpr uint32_t FORMAT_VERSION = 3;
constexpr char MAGIC[8] = {'L', 'B', 'M', 'K', 'P', 'T', 0, 0};
const char* RANK_FILE = "rank_0000_part_0000.bin";

[[noreturn]] void fail(const std::string& code, const std::string& msg) { throw Failure(code, msg); }

// ---- little-endian byte codec (solver.rs:1062-1109) ----------------------
void put(std::string& out, uint64_t v, int bytes) {
  for (int i = 0; i < bytes; ++i) out.push_back(char((v >> (8 * i)) & 0xff));
}
void put_f64(std::string& out, double v) {
  uint64_t b;
  std::memcpy(&b, &v, 8);
  put(out, b, 8);
}
// ---- FNV-1a 64 streams (solver.rs:831-859) --------------------------------
struct Hasher {
  uint64_t h = 0xcbf29ce484222325ull;
  void bytes(const void* d, size_t n) { h = fnv1a64(d, n, h); }
  void u64(uint64_t v) {
    unsigned char b[8];
    for (int i = 0; i < 8; ++i) b[i] = (v >> (8 * i)) & 0xff;
    bytes(b, 8);
  }
  void f64(double v) {
    uint64_t u;
    std::memcpy(&u, &v, 8);
    u64(u);
  }
  // hash_real: f32 runs hash the f32 bits (4 bytes), f64 runs the f64 bits.
  void real(double v, bool is64) {
    if (is64) {
      f64(v);
    } else {
      const float x = float(v);
      uint32_t u;
      std::memcpy(&u, &x, 4);
      unsigned char b[4];
      for (int i = 0; i < 4; ++i) b[i] = (u >> (8 * i)) & 0xff;
      bytes(b, 4);
    }
  }
};

// ---- halo-padded geometry (fields.rs:99-150; halo 1 on every axis) --------
struct Pad {
  int64_t nx, ny, nz, px, py, pz;
  explicit Pad(const Spec& s)
      : nx(s.dims[0]), ny(s.dims[1]), nz(s.dims[2]), px(nx + 2), py(ny + 2), pz(nz + 2) {}
  int64_t np() const { return px * py * pz; }
  int64_t nc() const { return nx * ny * nz; }
  int64_t pidx(int64_t x, int64_t y, int64_t z) const { return ((z + 1) * py + (y + 1)) * px + (x + 1); }
};

// Compact cell whose value the padded mask cell holds after the reference's
// mask exchange (halo.rs:457-492 over a monolithic part, subdomain.rs:31-44):
// periodic axes wrap (corners forwarded through the x, y, z phases); a halo
// cell behind a non-periodic face keeps the default (-1 here).
int64_t mask_source(const Spec& s, const Pad& g, int64_t x, int64_t y, int64_t z) {
  int64_t c[3] = {x, y, z};
  const int64_t n[3] = {g.nx, g.ny, g.nz};
  for (int a = 0; a < 3; ++a) {
    if (c[a] >= 0 && c[a] < n[a]) continue;
    if (!s.periodic[a]) return -1;
    c[a] = (c[a] + n[a]) % n[a];
  }
  return (c[2] * g.ny + c[1]) * g.nx + c[0];
}

void padded_masks(const Spec& s, const uint8_t* solid, const double* wall_u, std::vector<uint8_t>& ps,
                  std::vector<double>& pw) {
  const Pad g(s);
  ps.assign(size_t(g.np()), 0);
  pw.assign(size_t(3 * g.np()), 0.0);
  for (int64_t z = -1; z <= g.nz; ++z)
    for (int64_t y = -1; y <= g.ny; ++y)
      for (int64_t x = -1; x <= g.nx; ++x) {
        const int64_t src = mask_source(s, g, x, y, z);
        if (src < 0) continue;
        const int64_t p = g.pidx(x, y, z);
        ps[size_t(p)] = solid && solid[src] ? 1 : 0;
        if (wall_u)
          for (int k = 0; k < 3; ++k) pw[size_t(3 * p + k)] = wall_u[3 * src + k];
      }
}

const char* lattice_name(int q) { return q == 19 ? "D3Q19" : q == 27 ? "D3Q27" : "unknown"; }
int lattice_id(int q) { return q == 19 ? 319 : q == 27 ? 327 : 0; }
const char* dtype_name(bool f64) { return f64 ? "f64" : "f32"; }

// Q planes of a compact field into padded planes (halo zero), one padded
// row per append. The byte image is the host's: the format is little-endian
// and so are the hosts this library builds for.
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "checkpoint writer assumes a little-endian host");
template <class T>
void put_padded_t(std::string& out, const Pad& g, const double* v, int planes) {
  std::vector<T> row(size_t(g.px), T(0));
  const std::vector<T> zero(size_t(g.px), T(0));
  const size_t rb = size_t(g.px) * sizeof(T);
  for (int q = 0; q < planes; ++q)
    for (int64_t pz = 0; pz < g.pz; ++pz)
      for (int64_t py = 0; py < g.py; ++py) {
        const bool core_row = v && pz >= 1 && pz <= g.nz && py >= 1 && py <= g.ny;
        if (!core_row) {
          out.append(reinterpret_cast<const char*>(zero.data()), rb);
          continue;
        }
        const double* src = v + size_t(q) * size_t(g.nc()) + size_t(((pz - 1) * g.ny + (py - 1)) * g.nx);
        for (int64_t x = 0; x < g.nx; ++x) row[size_t(x + 1)] = T(src[x]);
        out.append(reinterpret_cast<const char*>(row.data()), rb);
      }
}
void put_padded(std::string& out, const Spec& s, const double* v, int planes, bool f64) {
  const Pad g(s);
  if (f64) put_padded_t<double>(out, g, v, planes);
  else put_padded_t<float>(out, g, v, planes);
}

// ---- JSON (serde_json::to_string_pretty layout; minimal reader) ------------
struct JVal {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  std::string text;  // number text or string value
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const std::string& k) const {
    for (auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  explicit JParser(const std::string& t) : s(t) {}
  [[noreturn]] void bad(const std::string& m) {
    fail("CKPT_MANIFEST_INVALID", m + " at byte " + std::to_string(i));
  }
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\n' || s[i] == '\r' || s[i] == '\t')) ++i;
  }
  bool lit(const char* w) {
    const size_t n = std::strlen(w);
    if (s.compare(i, n, w) == 0) {
      i += n;
      return true;
    }
    return false;
  }
  std::string str() {
    if (s[i] != '"') bad("expected string");
    ++i;
    std::string out;
    while (true) {
      if (i >= s.size()) bad("unterminated string");
      const char c = s[i++];
      if (c == '"') break;
      if (c != '\\') {
        out.push_back(c);
        continue;
      }
      if (i >= s.size()) bad("unterminated escape");
      const char e = s[i++];
      switch (e) {
        case '"': out.push_back('"'); break;
        case '\\': out.push_back('\\'); break;
        case '/': out.push_back('/'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'n': out.push_back('\n'); break;
        case 'r': out.push_back('\r'); break;
        case 't': out.push_back('\t'); break;
        case 'u': {
          if (i + 4 > s.size()) bad("short unicode escape");
          unsigned cp = 0;
          for (int k = 0; k < 4; ++k) {
            const char h = s[i + size_t(k)];
            const int d = h >= '0' && h <= '9' ? h - '0' : h >= 'a' && h <= 'f' ? h - 'a' + 10
                          : h >= 'A' && h <= 'F' ? h - 'A' + 10 : -1;
            if (d < 0) bad("bad unicode escape");
            cp = cp * 16 + unsigned(d);
          }
          i += 4;
          if (cp < 0x80) {
            out.push_back(char(cp));
          } else if (cp < 0x800) {
            out.push_back(char(0xc0 | (cp >> 6)));
            out.push_back(char(0x80 | (cp & 0x3f)));
          } else {
            out.push_back(char(0xe0 | (cp >> 12)));
            out.push_back(char(0x80 | ((cp >> 6) & 0x3f)));
            out.push_back(char(0x80 | (cp & 0x3f)));
          }
          break;
        }
        default: bad("bad escape");
      }
    }
    return out;
  }
  JVal value(int depth = 0) {
    if (depth > 64) bad("nesting too deep");
    ws();
    if (i >= s.size()) bad("unexpected end");
    JVal v;
    const char c = s[i];
    if (c == '{') {
      v.kind = JVal::OBJ;
      ++i;
      ws();
      if (s[i] == '}') {
        ++i;
        return v;
      }
      while (true) {
        ws();
        std::string k = str();
        ws();
        if (i >= s.size() || s[i] != ':') bad("expected ':'");
        ++i;
        v.obj.emplace_back(std::move(k), value(depth + 1));
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          break;
        }
        bad("expected ',' or '}'");
      }
    } else if (c == '[') {
      v.kind = JVal::ARR;
      ++i;
      ws();
      if (s[i] == ']') {
        ++i;
        return v;
      }
      while (true) {
        v.arr.push_back(value(depth + 1));
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          break;
        }
        bad("expected ',' or ']'");
      }
    } else if (c == '"') {
      v.kind = JVal::STR;
      v.text = str();
    } else if (lit("true")) {
      v.kind = JVal::BOOL;
      v.b = true;
    } else if (lit("false")) {
      v.kind = JVal::BOOL;
    } else if (lit("null")) {
      v.kind = JVal::NUL;
    } else {
      const size_t st = i;
      while (i < s.size() && (std::isdigit(static_cast<unsigned char>(s[i])) || s[i] == '-' || s[i] == '+' ||
                              s[i] == '.' || s[i] == 'e' || s[i] == 'E'))
        ++i;
      if (i == st) bad("unexpected character");
      v.kind = JVal::NUM;
      v.text = s.substr(st, i - st);
    }
    return v;
  }
};

// serde field access: a missing field or a value of the wrong type is a
// manifest error (the reference's From<serde_json::Error>, solver.rs:77-81).
const JVal& field(const JVal& o, const char* k) {
  const JVal* v = o.get(k);
  if (!v) fail("CKPT_MANIFEST_INVALID", std::string("missing field `") + k + "`");
  return *v;
}
uint64_t as_u64(const JVal& v, const char* k) {
  if (v.kind != JVal::NUM || v.text.empty() || v.text.find_first_not_of("0123456789") != std::string::npos)
    fail("CKPT_MANIFEST_INVALID", std::string("invalid type for `") + k + "`: expected an unsigned integer");
  errno = 0;
  const unsigned long long x = std::strtoull(v.text.c_str(), nullptr, 10);
  if (errno == ERANGE) fail("CKPT_MANIFEST_INVALID", std::string("integer out of range for `") + k + "`");
  return uint64_t(x);
}
const std::string& as_str(const JVal& v, const char* k) {
  if (v.kind != JVal::STR) fail("CKPT_MANIFEST_INVALID", std::string("invalid type for `") + k + "`: expected a string");
  return v.text;
}
std::vector<uint64_t> as_u64x3(const JVal& v, const char* k) {
  if (v.kind != JVal::ARR || v.arr.size() != 3)
    fail("CKPT_MANIFEST_INVALID", std::string("invalid type for `") + k + "`: expected an array of 3");
  return {as_u64(v.arr[0], k), as_u64(v.arr[1], k), as_u64(v.arr[2], k)};
}

// serde_json's f64 text for the manifest's `time` (an integer-valued f64
// prints with a trailing ".0").
std::string f64_text(double v) {
  char buf[64];
  if (v == std::floor(v) && std::fabs(v) < 1e16) {
    std::snprintf(buf, sizeof buf, "%.1f", v);
    return buf;
  }
  std::snprintf(buf, sizeof buf, "%.17g", v);
  return buf;
}

std::string arr3(uint64_t a, uint64_t b, uint64_t c, const std::string& ind) {
  return "[\n" + ind + "  " + std::to_string(a) + ",\n" + ind + "  " + std::to_string(b) + ",\n" + ind + "  " +
         std::to_string(c) + "\n" + ind + "]";
}

// checkpoint_manifest + write_checkpoint_manifest (solver.rs:4632-4670).
std::string manifest_text(const Spec& s, uint64_t step, uint64_t bytes, uint64_t payload_hash, uint64_t mhash,
                          bool stats) {
  std::string j = "{\n";
  j += "  \"kind\": \"lbmflow-checkpoint\",\n";
  j += "  \"format_version\": " + std::to_string(FORMAT_VERSION) + ",\n";
  j += "  \"step\": " + std::to_string(step) + ",\n";
  j += "  \"time\": " + f64_text(double(step)) + ",\n";
  j += "  \"dtype\": \"" + std::string(dtype_name(s.f64)) + "\",\n";
  j += "  \"lattice\": \"" + std::string(lattice_name(s.q)) + "\",\n";
  j += "  \"global\": " + arr3(uint64_t(s.dims[0]), uint64_t(s.dims[1]), uint64_t(s.dims[2]), "  ") + ",\n";
  j += "  \"scenario_hash\": \"" + hash_string(spec_hash(s)) + "\",\n";
  j += "  \"decomp_hash\": \"" + hash_string(decomp_hash(s)) + "\",\n";
  j += "  \"nranks\": 1,\n";
  j += "  \"ranks\": [\n";
  j += "    {\n";
  j += "      \"rank\": 0,\n";
  j += "      \"part\": 0,\n";
  j += "      \"file\": \"" + std::string(RANK_FILE) + "\",\n";
  j += "      \"origin\": " + arr3(0, 0, 0, "      ") + ",\n";
  j += "      \"core\": " + arr3(uint64_t(s.dims[0]), uint64_t(s.dims[1]), uint64_t(s.dims[2]), "      ") + ",\n";
  j += "      \"bytes\": " + std::to_string(bytes) + ",\n";
  j += "      \"payload_hash\": \"" + hash_string(payload_hash) + "\",\n";
  j += "      \"mask_hash\": \"" + hash_string(mhash) + "\"\n";
  j += "    }\n";
  j += "  ],\n";
  j += "  \"reserved\": {\n";
  j += "    \"particles\": false,\n";
  j += "    \"rng\": false,\n";
  j += std::string("    \"stats\": ") + (stats ? "true" : "false") + "\n";
  j += "  }\n";
  j += "}";
  return j;
}

std::string read_file(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) fail("CKPT_IO", "No such file or directory (os error 2): " + path);
  std::string b((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  if (in.bad()) fail("CKPT_IO", "read failed: " + path);
  return b;
}

void write_file(const std::string& path, const std::string& bytes) {
  std::ofstream out(path, std::ios::binary | std::ios::trunc);
  if (!out) fail("CKPT_IO", "cannot create " + path);
  out.write(bytes.data(), std::streamsize(bytes.size()));
  out.flush();
  if (!out) fail("CKPT_IO", "write failed: " + path);
}

// std::fs::create_dir_all
void make_dirs(const std::string& dir) {
  std::string cur;
  std::stringstream ss(dir);
  std::string part;
  if (!dir.empty() && dir[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part;
    if (::mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST) fail("CKPT_IO", "cannot create directory " + cur);
    struct stat sb;
    if (::stat(cur.c_str(), &sb) != 0 || !S_ISDIR(sb.st_mode)) fail("CKPT_IO", "not a directory: " + cur);
    cur += "/";
  }
}

std::string join(const std::string& dir, const std::string& f) {
  return dir.empty() ? f : (dir.back() == '/' ? dir + f : dir + "/" + f);
}

}  // namespace

bool json_object(const std::string& text) {
  try {
    JParser q(text);
    const JVal v = q.value();
    q.ws();
    return q.i == text.size() && v.kind == JVal::OBJ;
  } catch (const Failure&) {
    return false;
  }
}

// FNV-1a 64: h = (h ^ byte) * P per byte, mod 2^64. A zero byte leaves
// h ^ 0 = h, so a run of k zero bytes multiplies h by P^k; 64-byte blocks
// that are all zero (the stash planes, halo rows) take one multiply by P^64
// instead of 64 dependent steps. The result is the byte-serial hash.
namespace {
constexpr uint64_t FNV_PRIME = 0x100000001b3ull;
constexpr uint64_t prime_pow(int k) {
  uint64_t r = 1;
  for (int i = 0; i < k; ++i) r *= FNV_PRIME;
  return r;
}
constexpr uint64_t FNV_PRIME_64 = prime_pow(64);
}  // namespace

uint64_t fnv1a64(const void* data, size_t len, uint64_t h) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  size_t i = 0;
  for (; i + 64 <= len; i += 64) {
    uint64_t w[8];
    std::memcpy(w, p + i, 64);
    if ((w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) == 0) {
      h *= FNV_PRIME_64;
      continue;
    }
    for (int k = 0; k < 64; ++k) {
      h ^= p[i + size_t(k)];
      h *= FNV_PRIME;
    }
  }
  for (; i < len; ++i) {
    h ^= p[i];
    h *= FNV_PRIME;
  }
  return h;
}

std::string hash_string(uint64_t h) {
  char buf[40];
  std::snprintf(buf, sizeof buf, "fnv1a64:%016llx", static_cast<unsigned long long>(h));
  return buf;
}

// spec_hash (solver.rs:881-945) with every face closed and no sources or
// face patches.
uint64_t spec_hash(const Spec& s) {
  Hasher h;
  h.u64(3);
  h.u64(uint64_t(s.q));
  for (int a = 0; a < 3; ++a) h.u64(uint64_t(s.dims[a]));
  h.f64(s.nu);
  if (s.collision == LBMB_BGK) {
    h.u64(1);
  } else if (s.collision == LBMB_TRT) {
    h.u64(2);
    h.f64(s.magic);
  } else {
    h.u64(3);
    h.f64(s.omega_shear);
  }
  for (int a = 0; a < 3; ++a) h.u64(s.periodic[a] ? 1 : 0);
  for (int f = 0; f < 6; ++f) h.u64(0);  // FaceBC::Closed
  for (int a = 0; a < 3; ++a) h.real(s.force[a], s.f64);
  return h.h;
}

// decomp_hash (solver.rs:947-965) of the monolithic part: neighbours are
// Some(0) behind periodic faces (hashed 0 + 1) and None (0) elsewhere.
uint64_t decomp_hash(const Spec& s) {
  Hasher h;
  h.u64(1);
  for (int a = 0; a < 3; ++a) h.u64(s.periodic[a] ? 1 : 0);
  for (int a = 0; a < 3; ++a) h.u64(0);
  for (int a = 0; a < 3; ++a) h.u64(uint64_t(s.dims[a]));
  for (int f = 0; f < 6; ++f) h.u64(s.periodic[f / 2] ? 1 : 0);
  return h.h;
}

// part_mask_hash (solver.rs:967-979) over the padded masks.
uint64_t mask_hash(const Spec& s, const uint8_t* solid, const double* wall_u) {
  std::vector<uint8_t> ps;
  std::vector<double> pw;
  padded_masks(s, solid, wall_u, ps, pw);
  Hasher h;
  h.u64(ps.size());
  for (uint8_t v : ps) h.u64(v);
  for (double v : pw) h.real(v, s.f64);
  return h.h;
}

uint64_t padded_cells(const Spec& s) { return uint64_t(Pad(s).np()); }

Mapping::~Mapping() {
  if (p) ::munmap(const_cast<char*>(p), n);
}

std::string solid_section(const Spec& s, const uint8_t* solid) {
  std::vector<uint8_t> ps;
  std::vector<double> pw;
  padded_masks(s, solid, nullptr, ps, pw);
  return std::string(ps.begin(), ps.end());
}

uint64_t fnv1a64_zeros(uint64_t len, uint64_t h) {
  // k zero bytes multiply h by P^k (binary powering, mod 2^64)
  uint64_t r = 1, b = FNV_PRIME;
  for (uint64_t k = len; k; k >>= 1) {
    if (k & 1) r *= b;
    b *= b;
  }
  return h * r;
}

void append_reals(std::string& out, const double* v, size_t count, bool f64) {
  const size_t w = f64 ? 8 : 4;
  const size_t at = out.size();
  out.resize(at + count * w);
  char* d = &out[at];
  if (f64) {
    std::memcpy(d, v, count * 8);
  } else {
    for (size_t i = 0; i < count; ++i) {
      const float x = float(v[i]);
      std::memcpy(d + 4 * i, &x, 4);
    }
  }
}

void reals_to_double(const char* p, size_t count, bool f64, double* out) {
  if (f64) {
    std::memcpy(out, p, count * 8);
    return;
  }
  for (size_t i = 0; i < count; ++i) {
    float x;
    std::memcpy(&x, p + 4 * i, 4);
    out[i] = double(x);
  }
}

void unpad_to_double(const char* img, const Spec& s, int planes, double* out) {
  const Pad g(s);
  const size_t w = s.f64 ? 8 : 4;
  for (int q = 0; q < planes; ++q)
    for (int64_t z = 0; z < g.nz; ++z)
      for (int64_t y = 0; y < g.ny; ++y)
        reals_to_double(img + (size_t(q) * size_t(g.np()) + size_t(g.pidx(0, y, z))) * w, size_t(g.nx), s.f64,
                        out + size_t(q) * size_t(g.nc()) + size_t((z * g.ny + y) * g.nx));
}

// write_part_checkpoint + write_checkpoint_manifest (solver.rs:4536-4670)
// with the payload given as pieces. The rank file is written on a second
// thread while this one hashes the same pieces; zero pieces are written from
// a zero block and hashed as one multiply.
void write(const std::string& dir, const Spec& s, uint64_t step, const std::vector<SectionOut>& secs,
           const uint8_t* solid, const double* wall_u, bool stats) {
  if (s.q != 19 && s.q != 27) fail("CKPT_LATTICE_MISMATCH", "checkpoint lattice must be D3Q19 or D3Q27");
  const Pad g(s);
  std::string head;
  head.append(MAGIC, 8);
  put(head, FORMAT_VERSION, 4);
  head.push_back(0);
  head.push_back(s.f64 ? 1 : 0);
  put(head, uint64_t(lattice_id(s.q)), 2);
  put(head, uint64_t(s.q), 2);
  put(head, 3, 2);
  put(head, uint64_t(g.np()), 8);
  put(head, uint64_t(g.nc()), 8);
  put(head, secs.size(), 4);
  uint64_t off = 0;
  for (const SectionOut& e : secs) {
    uint64_t len = 0;
    for (const Piece& p : e.pieces) len += p.len;
    put(head, e.id, 4);
    put(head, off, 8);
    put(head, len, 8);
    off += len;
  }
  const uint64_t total = head.size() + off + 8;
  make_dirs(dir);
  const std::string path = join(dir, RANK_FILE);
  std::FILE* fh = std::fopen(path.c_str(), "wb");
  if (!fh) fail("CKPT_IO", "cannot create " + path);
  bool write_ok = true;
  struct Closer {  // closes the file if anything below throws
    std::FILE*& f;
    ~Closer() {
      if (f) std::fclose(f);
    }
  } closer{fh};
  std::thread writer([&] {
    static const std::vector<char> zeros(size_t(1) << 20, 0);  // zero runs shorter than 1 MB
    write_ok = std::fwrite(head.data(), 1, head.size(), fh) == head.size();
    for (const SectionOut& e : secs)
      for (const Piece& p : e.pieces) {
        if (!write_ok) return;
        if (p.data) {
          write_ok = std::fwrite(p.data, 1, size_t(p.len), fh) == size_t(p.len);
        } else if (p.len >= (uint64_t(1) << 20)) {
          // a long zero run is left as a hole (it reads back as zeros); the
          // trailer written after it sets the file's length
          write_ok = ::fseeko(fh, off_t(p.len), SEEK_CUR) == 0;
        } else {
          write_ok = std::fwrite(zeros.data(), 1, size_t(p.len), fh) == size_t(p.len);
        }
      }
  });
  uint64_t ph = 0xcbf29ce484222325ull;
  for (const SectionOut& e : secs)
    for (const Piece& p : e.pieces) ph = p.data ? fnv1a64(p.data, size_t(p.len), ph) : fnv1a64_zeros(p.len, ph);
  writer.join();
  std::string trailer;
  put(trailer, ph, 8);
  if (write_ok) write_ok = std::fwrite(trailer.data(), 1, 8, fh) == 8;
  if (std::fclose(fh) != 0) write_ok = false;
  fh = nullptr;
  if (!write_ok) fail("CKPT_IO", "write failed: " + path);
  write_file(join(dir, "manifest.json"), manifest_text(s, step, total, ph, mask_hash(s, solid, wall_u), stats));
}

void save(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u, const State& st) {
  if (s.q != 19 && s.q != 27) fail("CKPT_LATTICE_MISMATCH", "checkpoint lattice must be D3Q19 or D3Q27");
  const Pad g(s);
  const int64_t nc = g.nc(), np = g.np();
  if (int64_t(st.f.size()) != s.q * nc || int64_t(st.moments.size()) != 4 * nc ||
      (st.has_force_field && int64_t(st.force_field.size()) != 3 * nc))
    fail("CKPT_GEOM_MISMATCH", "state arrays differ from the checkpoint geometry");
  for (const Scalar& x : st.scalars)
    if ((x.q != 7 && x.q != s.q) || int64_t(x.h.size()) != x.q * nc || int64_t(x.conc.size()) != nc)
      fail("CKPT_GEOM_MISMATCH", "scalar arrays differ from the checkpoint geometry");
  const uint64_t w = s.f64 ? 8 : 4;
  std::vector<std::string> keep;  // storage of the pieces
  keep.reserve(16 + 4 * st.scalars.size());
  auto piece = [&](std::string b) {
    keep.push_back(std::move(b));
    return Piece{keep.back().data(), keep.back().size()};
  };
  std::vector<SectionOut> secs;
  {
    std::string b;
    put_padded(b, s, st.f.data(), s.q, s.f64);
    secs.push_back({SEC_F_PRIMARY, {piece(std::move(b))}});
  }
  secs.push_back({SEC_STALE_STASH, {Piece{nullptr, uint64_t(s.q) * uint64_t(np) * w}}});
  {
    std::string b;
    append_reals(b, st.moments.data(), st.moments.size(), s.f64);
    secs.push_back({SEC_MOMENTS, {piece(std::move(b))}});
  }
  secs.push_back({SEC_SOLID, {piece(solid_section(s, solid))}});
  if (st.has_force_field) {
    std::string b;
    append_reals(b, st.force_field.data(), st.force_field.size(), s.f64);
    secs.push_back({SEC_FORCE_FIELD, {piece(std::move(b))}});
  }
  if (!st.scalars.empty()) {
    SectionOut sec{SEC_SCALAR_FIELDS, {}};
    std::string count;
    put(count, st.scalars.size(), 4);
    sec.pieces.push_back(piece(std::move(count)));
    for (const Scalar& x : st.scalars) {
      std::string b;
      put_padded(b, s, x.h.data(), x.q, s.f64);
      sec.pieces.push_back(piece(scalar_head(x.name, x.diffusivity, uint64_t(x.q) * uint64_t(np))));
      sec.pieces.push_back(piece(std::move(b)));
      for (const Piece& p : scalar_tail(x.q, np, nc, w)) sec.pieces.push_back(p.data ? piece(std::string(p.data, p.len)) : p);
      std::string c;
      append_reals(c, x.conc.data(), x.conc.size(), s.f64);
      sec.pieces.push_back(piece(std::move(c)));
    }
    secs.push_back(std::move(sec));
  }
  if (st.has_qoi) secs.push_back({SEC_QOI_ACCUMULATORS, {piece(st.qoi_json)}});
  write(dir, s, st.step, secs, solid, wall_u, st.has_qoi);
}

// Scalar entry of the SCALAR_FIELDS section (solver.rs:1200-1217): name,
// diffusivity and the h length before the h planes ...
std::string scalar_head(const std::string& name, double diffusivity, uint64_t h_len) {
  std::string b;
  put(b, name.size(), 4);
  b += name;
  put_f64(b, diffusivity);
  put(b, h_len, 8);
  return b;
}
// ... then the ping-pong partner (zero planes) and the concentration
// length; the concentration values follow.
std::vector<Piece> scalar_tail(int q, int64_t np, int64_t nc, uint64_t w) {
  static thread_local std::string len_h, len_c;
  len_h.clear();
  put(len_h, uint64_t(q) * uint64_t(np), 8);
  len_c.clear();
  put(len_c, uint64_t(nc), 8);
  return {Piece{len_h.data(), 8}, Piece{nullptr, uint64_t(q) * uint64_t(np) * w}, Piece{len_c.data(), 8}};
}

// read_rank_file + load_into (solver.rs:1108-1198, 4759-5060).
View read(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u) {
  const Pad g(s);
  const int64_t nc = g.nc(), np = g.np();
  // load_into (solver.rs:4759-4824)
  const std::string text = read_file(join(dir, "manifest.json"));
  JParser jp(text);
  const JVal m = jp.value();
  jp.ws();
  if (jp.i != text.size()) jp.bad("trailing characters");
  if (m.kind != JVal::OBJ) fail("CKPT_MANIFEST_INVALID", "invalid type: expected struct CheckpointManifest");
  const std::string& kind = as_str(field(m, "kind"), "kind");
  const uint64_t fver = as_u64(field(m, "format_version"), "format_version");
  const uint64_t step = as_u64(field(m, "step"), "step");
  const JVal& tm = field(m, "time");
  if (tm.kind != JVal::NUM) fail("CKPT_MANIFEST_INVALID", "invalid type for `time`: expected f64");
  const std::string& dtype = as_str(field(m, "dtype"), "dtype");
  const std::string& lattice = as_str(field(m, "lattice"), "lattice");
  const std::vector<uint64_t> global = as_u64x3(field(m, "global"), "global");
  const std::string& scen = as_str(field(m, "scenario_hash"), "scenario_hash");
  const std::string& dech = as_str(field(m, "decomp_hash"), "decomp_hash");
  const uint64_t nranks = as_u64(field(m, "nranks"), "nranks");
  const JVal& ranks = field(m, "ranks");
  if (ranks.kind != JVal::ARR) fail("CKPT_MANIFEST_INVALID", "invalid type for `ranks`: expected a sequence");
  struct Entry {
    uint64_t rank, part;
    std::string file;
    std::vector<uint64_t> origin, core;
    uint64_t bytes;
    std::string payload_hash, mask_hash;
  };
  std::vector<Entry> entries;
  for (const JVal& r : ranks.arr) {
    if (r.kind != JVal::OBJ) fail("CKPT_MANIFEST_INVALID", "invalid type: expected struct CheckpointRank");
    entries.push_back({as_u64(field(r, "rank"), "rank"), as_u64(field(r, "part"), "part"),
                       as_str(field(r, "file"), "file"), as_u64x3(field(r, "origin"), "origin"),
                       as_u64x3(field(r, "core"), "core"), as_u64(field(r, "bytes"), "bytes"),
                       as_str(field(r, "payload_hash"), "payload_hash"), as_str(field(r, "mask_hash"), "mask_hash")});
  }
  const JVal& reserved = field(m, "reserved");
  if (reserved.kind != JVal::OBJ) fail("CKPT_MANIFEST_INVALID", "invalid type for `reserved`: expected a map");
  for (auto& kv : reserved.obj)
    if (kv.second.kind != JVal::BOOL) fail("CKPT_MANIFEST_INVALID", "invalid type for `reserved`: expected bool");

  if (kind != "lbmflow-checkpoint") fail("CKPT_BAD_MAGIC", "manifest kind is " + kind);
  if (fver != FORMAT_VERSION)
    fail("CKPT_VERSION_MISMATCH",
         "checkpoint format_version " + std::to_string(fver) + " differs from supported " +
             std::to_string(FORMAT_VERSION) +
             "; rerun from the original scenario or migrate with a checkpoint upgrader before restart");
  if (dtype != dtype_name(s.f64))
    fail("CKPT_DTYPE_MISMATCH", "checkpoint dtype " + dtype + " differs from run dtype " + dtype_name(s.f64));
  if (lattice != lattice_name(s.q))
    fail("CKPT_LATTICE_MISMATCH",
         "checkpoint lattice " + lattice + " differs from run lattice " + lattice_name(s.q));
  auto dims_text = [](uint64_t a, uint64_t b, uint64_t c) {
    return "[" + std::to_string(a) + ", " + std::to_string(b) + ", " + std::to_string(c) + "]";
  };
  if (global[0] != uint64_t(s.dims[0]) || global[1] != uint64_t(s.dims[1]) || global[2] != uint64_t(s.dims[2]))
    fail("CKPT_GEOM_MISMATCH", "checkpoint global " + dims_text(global[0], global[1], global[2]) +
                                   " differs from run " + dims_text(uint64_t(s.dims[0]), uint64_t(s.dims[1]),
                                                                    uint64_t(s.dims[2])));
  const std::string expected = hash_string(spec_hash(s));
  if (scen != expected)
    fail("CKPT_SCENARIO_MISMATCH", "scenario_hash differed: checkpoint=" + scen + " current=" + expected);
  // load_into_with_layout (solver.rs:4895-5060)
  const std::string cur_dec = hash_string(decomp_hash(s));
  if (dech != cur_dec) fail("CKPT_DECOMP_MISMATCH", "decomp_hash differed: checkpoint=" + dech + " current=" + cur_dec);
  if (nranks != 1)
    fail("CKPT_RANK_MISMATCH", "checkpoint rank count " + std::to_string(nranks) + " differs from current 1");
  std::vector<const Entry*> mine;
  for (auto& e : entries)
    if (e.rank == 0) mine.push_back(&e);
  if (mine.size() != 1)
    fail("CKPT_DECOMP_MISMATCH", "checkpoint has " + std::to_string(mine.size()) +
                                     " payload parts for rank 0, current owner has 1");
  const Entry& e = *mine[0];
  if (e.origin[0] || e.origin[1] || e.origin[2] || e.core[0] != uint64_t(s.dims[0]) ||
      e.core[1] != uint64_t(s.dims[1]) || e.core[2] != uint64_t(s.dims[2]))
    fail("CKPT_GEOM_MISMATCH", "part geometry differed: checkpoint rank=0 part=" + std::to_string(e.part) +
                                   " origin=" + dims_text(e.origin[0], e.origin[1], e.origin[2]) + " core=" +
                                   dims_text(e.core[0], e.core[1], e.core[2]) + ", current origin=[0, 0, 0] core=" +
                                   dims_text(uint64_t(s.dims[0]), uint64_t(s.dims[1]), uint64_t(s.dims[2])));
  const std::string cur_mask = hash_string(mask_hash(s, solid, wall_u));
  if (e.mask_hash != cur_mask)
    fail("CKPT_MASK_MISMATCH", "mask_hash differed for rank=0 part=" + std::to_string(e.part) +
                                   ": checkpoint=" + e.mask_hash + " current=" + cur_mask);

  // read_rank_file (solver.rs:1108-1198): the file is mapped (no copy; a
  // checkpoint just written is served from the page cache) and the payload
  // hashed in place.
  if (e.file.find('/') != std::string::npos || e.file == ".." || e.file.empty())
    fail("CKPT_MANIFEST_INVALID", "rank file name must be a plain file name: " + e.file);
  const std::string path = join(dir, e.file);
  auto map = std::make_shared<Mapping>();
  {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) fail("CKPT_IO", "No such file or directory (os error 2): " + path);
    struct stat sb;
    if (::fstat(fd, &sb) != 0) {
      ::close(fd);
      fail("CKPT_IO", "cannot stat " + path);
    }
    map->n = size_t(sb.st_size);
    if (map->n > 0) {
      void* p = ::mmap(nullptr, map->n, PROT_READ, MAP_PRIVATE, fd, 0);
      if (p == MAP_FAILED) {
        ::close(fd);
        fail("CKPT_IO", "cannot map " + path);
      }
      map->p = static_cast<const char*>(p);
      ::madvise(p, map->n, MADV_SEQUENTIAL);
      ::madvise(p, map->n, MADV_WILLNEED);
    }
    ::close(fd);
  }
  const char* buf = map->p;
  const size_t fsize = map->n;
  // header and section table
  size_t pos = 0;
  auto take = [&](size_t k) -> const char* {
    if (pos > fsize || fsize - pos < k)
      fail("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload");
    const char* p = buf + pos;
    pos += k;
    return p;
  };
  auto uint = [&](int bytes) {
    const unsigned char* p = reinterpret_cast<const unsigned char*>(take(size_t(bytes)));
    uint64_t v = 0;
    for (int i = 0; i < bytes; ++i) v |= uint64_t(p[i]) << (8 * i);
    return v;
  };
  if (std::memcmp(take(8), MAGIC, 8) != 0) fail("CKPT_BAD_MAGIC", "rank file magic is not LBMKPT");
  const uint64_t rv = uint(4);
  if (rv != FORMAT_VERSION)
    fail("CKPT_VERSION_MISMATCH",
         "rank file format_version " + std::to_string(rv) + " differs from supported " +
             std::to_string(FORMAT_VERSION) +
             "; rerun from the original scenario or migrate with a checkpoint upgrader before restart");
  if (uint(1) != 0) fail("CKPT_BAD_MAGIC", "cross-endian checkpoints are not supported by this checkpoint format");
  const uint64_t hdtype = uint(1), hlat = uint(2), hq = uint(2), hd = uint(2);
  const uint64_t hnp = uint(8), hnc = uint(8);
  const uint64_t nsec = uint(4);
  struct Sec {
    uint64_t id, off, len;
  };
  std::vector<Sec> table;
  for (uint64_t k = 0; k < nsec; ++k) {
    Sec t;
    t.id = uint(4);
    t.off = uint(8);
    t.len = uint(8);
    table.push_back(t);
  }
  if (fsize - pos < 8) fail("CKPT_TRUNCATED", "rank file is missing payload hash trailer");
  const size_t pend = fsize - 8;
  const char* payload = buf + pos;
  const size_t plen = pend - pos;
  const uint64_t ph_calc = fnv1a64(payload, plen);
  uint64_t phash = 0;
  for (int i = 0; i < 8; ++i) phash |= uint64_t(static_cast<unsigned char>(buf[pend + size_t(i)])) << (8 * i);
  if (ph_calc != phash) fail("CKPT_PAYLOAD_CORRUPT", "rank file payload hash does not match its contents");
  std::map<uint32_t, std::pair<size_t, size_t>> sections;  // id -> (offset, length); later entries win
  for (const Sec& t : table) {
    if (t.off > plen || t.len > plen - t.off)
      fail("CKPT_TRUNCATED", "section " + std::to_string(t.id) + " range " + std::to_string(t.off) + ".." +
                                 std::to_string(t.off + t.len) + " exceeds payload length " + std::to_string(plen));
    sections[uint32_t(t.id)] = {size_t(t.off), size_t(t.len)};
  }
  if (hdtype != (s.f64 ? 1u : 0u)) fail("CKPT_DTYPE_MISMATCH", "rank file dtype differs from requested run precision");
  if (hlat != uint64_t(lattice_id(s.q)) || hq != uint64_t(s.q) || hd != 3)
    fail("CKPT_LATTICE_MISMATCH", "rank file lattice metadata differs from requested lattice");
  if (hnp != uint64_t(np) || hnc != uint64_t(nc))
    fail("CKPT_GEOM_MISMATCH", "rank file np/n_core " + std::to_string(hnp) + "/" + std::to_string(hnc) +
                                   " differs from current " + std::to_string(np) + "/" + std::to_string(nc));
  if (hash_string(phash) != e.payload_hash)
    fail("CKPT_PAYLOAD_CORRUPT",
         "rank payload hash " + hash_string(phash) + " differs from manifest " + e.payload_hash);
  auto section = [&](uint32_t id) -> const std::pair<size_t, size_t>* {
    auto it = sections.find(id);
    return it == sections.end() ? nullptr : &it->second;
  };
  auto required = [&](uint32_t id, const char* name) {
    const auto* p = section(id);
    if (!p) fail("CKPT_TRUNCATED", std::string("checkpoint is missing required section ") + name);
    return *p;
  };
  const size_t w = s.f64 ? 8 : 4;
  auto check_len = [&](size_t len, size_t expected) {
    if (len != expected * w)
      fail("CKPT_GEOM_MISMATCH", "section length " + std::to_string(len) + " does not match expected " +
                                     std::to_string(expected) + " values of " + std::to_string(w) + " bytes");
  };
  View v;
  v.hold = map;
  v.step = step;
  {
    const auto p = required(SEC_F_PRIMARY, "F_PRIMARY");
    check_len(p.second, size_t(s.q) * size_t(np));
    v.f = payload + p.first;
    const auto t = required(SEC_STALE_STASH, "STALE_STASH");
    check_len(t.second, size_t(s.q) * size_t(np));
    const auto mo = required(SEC_MOMENTS, "MOMENTS");
    check_len(mo.second, size_t(4 * nc));
    v.moments = payload + mo.first;
  }
  if (const auto* p = section(SEC_SOLID)) {
    if (p->second != size_t(np))
      fail("CKPT_GEOM_MISMATCH", "solid section length differs from current padded geometry");
    std::vector<uint8_t> ps;
    std::vector<double> pw;
    padded_masks(s, solid, wall_u, ps, pw);
    for (size_t i = 0; i < size_t(np); ++i)
      if ((payload[p->first + i] != 0) != (ps[i] != 0))
        fail("CKPT_MASK_MISMATCH", "serialized solid mask differs from rebuilt mask");
  }
  if (const auto* p = section(SEC_FORCE_FIELD)) {
    check_len(p->second, size_t(3 * nc));
    v.force_field = payload + p->first;
  }
  if (const auto* p = section(SEC_SCALAR_FIELDS)) {
    // restore_scalar_checkpoint (solver.rs:1219-1287). The reference's
    // scalars live on the hydro lattice; a D3Q7 scalar (7 planes) is read too.
    const char* base = payload + p->first;
    const size_t blen = p->second;
    size_t at = 0;
    auto stake = [&](size_t k) -> const char* {
      if (at > blen || blen - at < k) fail("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload");
      const char* r = base + at;
      at += k;
      return r;
    };
    auto suint = [&](int bytes) {
      const unsigned char* q = reinterpret_cast<const unsigned char*>(stake(size_t(bytes)));
      uint64_t x = 0;
      for (int i = 0; i < bytes; ++i) x |= uint64_t(q[i]) << (8 * i);
      return x;
    };
    const uint64_t count = suint(4);
    for (uint64_t k = 0; k < count; ++k) {
      ScalarView x;
      const uint64_t nl = suint(4);
      x.name.assign(stake(size_t(nl)), size_t(nl));
      const uint64_t db = suint(8);
      std::memcpy(&x.diffusivity, &db, 8);
      const uint64_t hl = suint(8);
      if (hl > blen) fail("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload");
      x.h = stake(size_t(hl) * w);
      const uint64_t tl = suint(8);
      if (tl > blen) fail("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload");
      stake(size_t(tl) * w);
      const uint64_t cl = suint(8);
      if (cl > blen) fail("CKPT_TRUNCATED", "rank file ended before the declared header/table/payload");
      x.conc = stake(size_t(cl) * w);
      const bool q_ok = hl % uint64_t(np) == 0 && (hl / uint64_t(np) == 7 || hl / uint64_t(np) == uint64_t(s.q));
      if (!q_ok || tl != hl || cl != uint64_t(nc))
        fail("CKPT_GEOM_MISMATCH", "scalar checkpoint section length differs from current geometry");
      x.q = int(hl / uint64_t(np));
      v.scalars.push_back(std::move(x));
    }
    if (at != blen) fail("CKPT_PAYLOAD_CORRUPT", "scalar checkpoint section has trailing bytes");
  }
  if (section(SEC_PHASE_FIELD))
    fail("CKPT_UNSUPPORTED", "the checkpoint carries a phase-field distribution; this solver is single-phase");
  if (const auto* p = section(SEC_QOI_ACCUMULATORS)) {
    v.has_qoi = true;
    v.qoi_json.assign(payload + p->first, p->second);
    if (!json_object(v.qoi_json)) fail("CKPT_MANIFEST_INVALID", "QOI accumulator section is not a JSON object");
  }
  return v;
}

State load(const std::string& dir, const Spec& s, const uint8_t* solid, const double* wall_u) {
  const Pad g(s);
  const size_t nc = size_t(g.nc());
  const View v = read(dir, s, solid, wall_u);
  State st;
  st.step = v.step;
  st.f.resize(size_t(s.q) * nc);
  unpad_to_double(v.f, s, s.q, st.f.data());
  st.moments.resize(4 * nc);
  reals_to_double(v.moments, 4 * nc, s.f64, st.moments.data());
  if (v.force_field) {
    st.has_force_field = true;
    st.force_field.resize(3 * nc);
    reals_to_double(v.force_field, 3 * nc, s.f64, st.force_field.data());
  }
  for (const ScalarView& x : v.scalars) {
    Scalar y;
    y.name = x.name;
    y.diffusivity = x.diffusivity;
    y.q = x.q;
    y.h.resize(size_t(x.q) * nc);
    unpad_to_double(x.h, s, x.q, y.h.data());
    y.conc.resize(nc);
    reals_to_double(x.conc, nc, s.f64, y.conc.data());
    st.scalars.push_back(std::move(y));
  }
  st.has_qoi = v.has_qoi;
  st.qoi_json = v.qoi_json;
  return st;
}

Spec spec_of(const lbmb_config& c) {
  Spec s;
  s.q = c.lattice;
  s.collision = c.collision;
  s.f64 = c.storage == LBMB_STORE_F64;
  for (int a = 0; a < 3; ++a) {
    s.dims[a] = c.dims[a];
    s.periodic[a] = c.periodic[a] != 0;
    s.force[a] = c.force[a];
  }
  s.nu = c.nu;
  s.magic = c.magic;
  s.omega_shear = c.omega_shear;
  return s;
}

}  // namespace ckpt
}  // namespace lbmb

// ---------------------------------------------------------------------------
// Host-only C ABI: the format on caller-owned compact arrays (no device).
// ---------------------------------------------------------------------------
namespace {

lbmb::ckpt::Spec to_spec(const lbmb_checkpoint_spec& c) {
  if (c.lattice != 19 && c.lattice != 27) throw lbmb::ckpt::Failure("CKPT_LATTICE_MISMATCH", "lattice must be 19 or 27");
  if (c.dtype_bits != 32 && c.dtype_bits != 64)
    throw lbmb::ckpt::Failure("CKPT_DTYPE_MISMATCH", "dtype_bits must be 32 or 64");
  for (int a = 0; a < 3; ++a)
    if (c.dims[a] < 1) throw lbmb::ckpt::Failure("CKPT_GEOM_MISMATCH", "dims must be positive");
  lbmb::ckpt::Spec s;
  s.q = c.lattice;
  s.collision = c.collision;
  s.f64 = c.dtype_bits == 64;
  for (int a = 0; a < 3; ++a) {
    s.dims[a] = c.dims[a];
    s.periodic[a] = c.periodic[a] != 0;
    s.force[a] = c.force[a];
  }
  s.nu = c.nu;
  s.magic = c.magic;
  s.omega_shear = c.omega_shear;
  return s;
}

template <class F>
int host_guarded(F&& fn) {
  try {
    fn();
    lbmb::g_last_error.clear();
    return LBMB_OK;
  } catch (const lbmb::ckpt::Failure& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_CHECKPOINT;
  } catch (const std::bad_alloc&) {
    lbmb::g_last_error = "host allocation failed";
    return LBMB_ERR_NOMEM;
  } catch (const std::exception& e) {
    lbmb::g_last_error = e.what();
    return LBMB_ERR_INVALID;
  }
}

}  // namespace

extern "C" {

uint64_t lbmb_fnv1a64(const void* data, uint64_t len) { return lbmb::ckpt::fnv1a64(data, size_t(len)); }

int lbmb_checkpoint_write_host(const char* dir, const lbmb_checkpoint_spec* spec, const uint8_t* solid,
                               const double* wall_u, const lbmb_checkpoint_data* data) {
  return host_guarded([&] {
    if (!dir || !spec || !data || !data->f || !data->moments)
      throw std::invalid_argument("null argument");
    const lbmb::ckpt::Spec s = to_spec(*spec);
    const size_t n = size_t(s.dims[0]) * size_t(s.dims[1]) * size_t(s.dims[2]);
    lbmb::ckpt::State st;
    st.step = data->step;
    st.f.assign(data->f, data->f + size_t(s.q) * n);
    st.moments.assign(data->moments, data->moments + 4 * n);
    st.has_force_field = data->has_force_field != 0;
    if (st.has_force_field) {
      if (!data->force_field) throw std::invalid_argument("null force field");
      st.force_field.assign(data->force_field, data->force_field + 3 * n);
    }
    if (data->n_scalars < 0 || (data->n_scalars > 0 && !data->scalars)) throw std::invalid_argument("bad scalar list");
    for (int32_t k = 0; k < data->n_scalars; ++k) {
      const lbmb_checkpoint_scalar& c = data->scalars[k];
      if (!c.h || !c.conc) throw std::invalid_argument("null scalar array");
      lbmb::ckpt::Scalar x;
      x.name.assign(c.name, strnlen(c.name, sizeof c.name));
      x.diffusivity = c.diffusivity;
      x.q = c.q;
      x.h.assign(c.h, c.h + size_t(c.q) * n);
      x.conc.assign(c.conc, c.conc + n);
      st.scalars.push_back(std::move(x));
    }
    st.has_qoi = data->has_qoi != 0;
    if (st.has_qoi) {
      if (!data->qoi_json || data->qoi_len < 0) throw std::invalid_argument("bad QOI JSON");
      st.qoi_json.assign(data->qoi_json, size_t(data->qoi_len));
    }
    lbmb::ckpt::save(dir, s, solid, wall_u, st);
  });
}

int lbmb_checkpoint_read_host(const char* dir, const lbmb_checkpoint_spec* spec, const uint8_t* solid,
                              const double* wall_u, lbmb_checkpoint_data* data) {
  return host_guarded([&] {
    if (!dir || !spec || !data || !data->f || !data->moments) throw std::invalid_argument("null argument");
    const lbmb::ckpt::Spec s = to_spec(*spec);
    const size_t n = size_t(s.dims[0]) * size_t(s.dims[1]) * size_t(s.dims[2]);
    const lbmb::ckpt::State st = lbmb::ckpt::load(dir, s, solid, wall_u);
    if (int64_t(st.scalars.size()) > int64_t(data->scalar_capacity))
      throw lbmb::ckpt::Failure("CKPT_GEOM_MISMATCH", "more scalar distributions than the caller's capacity");
    for (size_t k = 0; k < st.scalars.size(); ++k) {
      const lbmb_checkpoint_scalar& c = data->scalars[k];
      if (!c.h || !c.conc || c.h_capacity < int64_t(st.scalars[k].h.size()) ||
          st.scalars[k].name.size() >= sizeof c.name)
        throw lbmb::ckpt::Failure("CKPT_GEOM_MISMATCH", "scalar buffers smaller than the checkpoint's");
    }
    if (st.has_qoi && (!data->qoi_json || data->qoi_capacity < int64_t(st.qoi_json.size())))
      throw lbmb::ckpt::Failure("CKPT_GEOM_MISMATCH", "QOI buffer smaller than the checkpoint's");
    if (st.has_force_field && !data->force_field) throw std::invalid_argument("null force field");
    data->step = st.step;
    std::memcpy(data->f, st.f.data(), size_t(s.q) * n * sizeof(double));
    std::memcpy(data->moments, st.moments.data(), 4 * n * sizeof(double));
    data->has_force_field = st.has_force_field ? 1 : 0;
    if (st.has_force_field) std::memcpy(data->force_field, st.force_field.data(), 3 * n * sizeof(double));
    data->n_scalars = int32_t(st.scalars.size());
    for (size_t k = 0; k < st.scalars.size(); ++k) {
      lbmb_checkpoint_scalar& c = data->scalars[k];
      std::memset(c.name, 0, sizeof c.name);
      std::memcpy(c.name, st.scalars[k].name.data(), st.scalars[k].name.size());
      c.diffusivity = st.scalars[k].diffusivity;
      c.q = st.scalars[k].q;
      std::memcpy(c.h, st.scalars[k].h.data(), st.scalars[k].h.size() * sizeof(double));
      std::memcpy(c.conc, st.scalars[k].conc.data(), n * sizeof(double));
    }
    data->has_qoi = st.has_qoi ? 1 : 0;
    data->qoi_len = int64_t(st.qoi_json.size());
    if (st.has_qoi) std::memcpy(data->qoi_json, st.qoi_json.data(), st.qoi_json.size());
  });
}

}  // extern "C"
