// .taas v2 container: writer, reader, inspector (host code).
// crates/SiMuse/crates/taas-format/src/{types,writer,reader,inspect,lib}.rs
#include "taas.h"

#include <dlfcn.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <algorithm>
#include <stdexcept>
#include <thread>

namespace sg {
namespace taas {

// ---------------------------------------------------------------------------
// CRC-32 (IEEE 802.3, reflected polynomial 0xEDB88320, initial and final
// complement), the checksum crc32fast computes (writer.rs:6-10); eight bytes
// per table round (slicing-by-8: table k advances a byte's remainder through
// k further zero bytes)
// ---------------------------------------------------------------------------
static uint32_t crc32_serial(const uint8_t *p, size_t n) {
  static const auto T = [] {
    std::vector<uint32_t> t(8 * 256);
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
      t[i] = c;
    }
    for (int k = 1; k < 8; ++k)
      for (uint32_t i = 0; i < 256; ++i) t[k * 256 + i] = (t[(k - 1) * 256 + i] >> 8) ^ t[t[(k - 1) * 256 + i] & 0xFFu];
    return t;
  }();
  const uint32_t *t = T.data();
  uint32_t c = 0xFFFFFFFFu;
  for (; n >= 8; p += 8, n -= 8) {
    uint32_t lo, hi;
    std::memcpy(&lo, p, 4);  // little-endian host
    std::memcpy(&hi, p + 4, 4);
    lo ^= c;
    c = t[7 * 256 + (lo & 0xFFu)] ^ t[6 * 256 + ((lo >> 8) & 0xFFu)] ^ t[5 * 256 + ((lo >> 16) & 0xFFu)] ^
        t[4 * 256 + (lo >> 24)] ^ t[3 * 256 + (hi & 0xFFu)] ^ t[2 * 256 + ((hi >> 8) & 0xFFu)] ^
        t[1 * 256 + ((hi >> 16) & 0xFFu)] ^ t[hi >> 24];
  }
  for (; n; ++p, --n) c = t[(c ^ *p) & 0xFFu] ^ (c >> 8);
  return c ^ 0xFFFFFFFFu;
}

// Polynomials over GF(2) modulo the CRC polynomial, in the reflected bit
// order of the remainder (bit 31 = x^0): a*b mod P.
static uint32_t gf2_mulmod(uint32_t a, uint32_t b) {
  uint32_t prod = 0;
  for (uint32_t m = 1u << 31; m; m >>= 1) {
    if (a & m) prod ^= b;
    b = (b & 1u) ? (b >> 1) ^ 0xEDB88320u : b >> 1;  // b *= x
  }
  return prod;
}

// CRC of A||B from crc(A), crc(B) and |B|: crc(A) times x^(8|B|) mod P, plus
// crc(B) (the pre and post conditioning cancel between the two).
static uint32_t crc32_combine(uint32_t ca, uint32_t cb, uint64_t nb) {
  uint32_t xp = 1u << 31;  // x^0
  uint32_t sq = 1u << 30;  // x^1, squared below to x^(2^k)
  for (uint64_t e = nb * 8; e; e >>= 1) {
    if (e & 1u) xp = gf2_mulmod(xp, sq);
    sq = gf2_mulmod(sq, sq);
  }
  return gf2_mulmod(ca, xp) ^ cb;
}

uint32_t crc32(const uint8_t *p, size_t n) {
  const size_t min_chunk = 4u << 20;
  unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  T = (unsigned)std::min<size_t>(T, n / min_chunk);
  if (T <= 1) return crc32_serial(p, n);
  std::vector<uint32_t> c(T);
  std::vector<size_t> len(T);
  std::vector<std::thread> th;
  const size_t chunk = n / T;
  for (unsigned k = 0; k < T; ++k) {
    const size_t a = k * chunk;
    len[k] = k + 1 == T ? n - a : chunk;
    th.emplace_back([&, k, a] { c[k] = crc32_serial(p + a, len[k]); });
  }
  for (auto &x : th) x.join();
  uint32_t r = c[0];
  for (unsigned k = 1; k < T; ++k) r = crc32_combine(r, c[k], len[k]);
  return r;
}

// types.rs:58-67
size_t kind_size(const std::string &k) {
  if (k == "f32" || k == "i32") return 4;
  if (k == "i64" || k == "u64") return 8;
  if (k == "u8") return 1;
  return 0;
}

static bool kind_known(const std::string &k) {
  return kind_size(k) || k == "str" || k == "json" || k == "blob";
}

// ---------------------------------------------------------------------------
// zstd through the system library's public one-shot API
// ---------------------------------------------------------------------------
namespace {
struct Zstd {
  void *h = nullptr;
  size_t (*compress)(void *, size_t, const void *, size_t, int) = nullptr;
  size_t (*bound)(size_t) = nullptr;
  unsigned (*is_error)(size_t) = nullptr;
  size_t (*decompress)(void *, size_t, const void *, size_t) = nullptr;
  unsigned long long (*content_size)(const void *, size_t) = nullptr;
};
const Zstd *zstd() {
  static Zstd z = [] {
    Zstd r;
    r.h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
    if (!r.h) return r;
    r.compress = (decltype(r.compress))dlsym(r.h, "ZSTD_compress");
    r.bound = (decltype(r.bound))dlsym(r.h, "ZSTD_compressBound");
    r.is_error = (decltype(r.is_error))dlsym(r.h, "ZSTD_isError");
    r.decompress = (decltype(r.decompress))dlsym(r.h, "ZSTD_decompress");
    r.content_size = (decltype(r.content_size))dlsym(r.h, "ZSTD_getFrameContentSize");
    if (!r.compress || !r.bound || !r.is_error || !r.decompress || !r.content_size) r.h = nullptr;
    return r;
  }();
  return z.h ? &z : nullptr;
}
}  // namespace

bool zstd_available() { return zstd() != nullptr; }

// ---------------------------------------------------------------------------
// JSON: the manifest as serde_json writes it (compact, struct field order,
// None fields skipped, BTreeMap keys sorted) and a small parser for reading
// ---------------------------------------------------------------------------
static void json_str(std::string &o, const std::string &s) {
  static const char *hex = "0123456789abcdef";
  o += '"';
  for (unsigned char c : s) {
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\b': o += "\\b"; break;
      case '\f': o += "\\f"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      default:
        if (c < 0x20) {
          o += "\\u00";
          o += hex[c >> 4];
          o += hex[c & 15];
        } else {
          o += (char)c;
        }
    }
  }
  o += '"';
}

static std::string manifest_json(const Manifest &m) {
  std::string o = "{\"version\":";
  json_str(o, m.version);
  o += ",\"created\":";
  json_str(o, m.created);
  if (m.has_game) {
    o += ",\"game\":";
    json_str(o, m.game);
  }
  o += ",\"sections\":[";
  for (size_t i = 0; i < m.sections.size(); ++i) {
    const Section &s = m.sections[i];
    if (i) o += ',';
    o += "{\"name\":";
    json_str(o, s.name);
    o += ",\"kind\":";
    json_str(o, s.kind);
    o += ",\"count\":" + std::to_string(s.count) + ",\"offset\":" + std::to_string(s.offset) +
         ",\"size\":" + std::to_string(s.size);
    if (s.has_crc) o += ",\"crc32\":" + std::to_string(s.crc);
    if (!s.compression.empty()) {
      o += ",\"compression\":";
      json_str(o, s.compression);
    }
    if (s.has_usize) o += ",\"uncompressed_size\":" + std::to_string(s.usize);
    o += '}';
  }
  o += "],\"metadata\":{";
  bool first = true;
  for (auto &kv : m.metadata) {
    if (!first) o += ',';
    first = false;
    json_str(o, kv.first);
    o += ':';
    json_str(o, kv.second);
  }
  o += "}}";
  return o;
}

namespace {
struct JVal {
  enum T { Null, Bool, Num, Str, Arr, Obj } t = Null;
  bool b = false;
  bool is_uint = false;
  uint64_t u = 0;
  double d = 0;
  std::string s;
  std::vector<JVal> a;
  std::vector<std::pair<std::string, JVal>> o;
  const JVal *get(const std::string &k) const {
    for (auto &kv : o)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct JParser {
  const char *p, *e;
  [[noreturn]] void fail(const char *what) { throw std::runtime_error(std::string("Invalid manifest JSON: ") + what); }
  void ws() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  void put_utf8(std::string &o, uint32_t cp) {
    if (cp < 0x80) o += (char)cp;
    else if (cp < 0x800) {
      o += (char)(0xC0 | (cp >> 6));
      o += (char)(0x80 | (cp & 0x3F));
    } else if (cp < 0x10000) {
      o += (char)(0xE0 | (cp >> 12));
      o += (char)(0x80 | ((cp >> 6) & 0x3F));
      o += (char)(0x80 | (cp & 0x3F));
    } else {
      o += (char)(0xF0 | (cp >> 18));
      o += (char)(0x80 | ((cp >> 12) & 0x3F));
      o += (char)(0x80 | ((cp >> 6) & 0x3F));
      o += (char)(0x80 | (cp & 0x3F));
    }
  }
  uint32_t hex4() {
    if (e - p < 4) fail("truncated \\u escape");
    uint32_t v = 0;
    for (int k = 0; k < 4; ++k) {
      const char c = *p++;
      v <<= 4;
      if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
      else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
      else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
      else fail("bad \\u escape");
    }
    return v;
  }
  std::string str() {
    if (p >= e || *p != '"') fail("expected a string");
    ++p;
    std::string o;
    while (true) {
      if (p >= e) fail("unterminated string");
      const char c = *p++;
      if (c == '"') break;
      if ((unsigned char)c < 0x20) fail("control character in string");
      if (c != '\\') {
        o += c;
        continue;
      }
      if (p >= e) fail("unterminated escape");
      const char x = *p++;
      switch (x) {
        case '"': o += '"'; break;
        case '\\': o += '\\'; break;
        case '/': o += '/'; break;
        case 'b': o += '\b'; break;
        case 'f': o += '\f'; break;
        case 'n': o += '\n'; break;
        case 'r': o += '\r'; break;
        case 't': o += '\t'; break;
        case 'u': {
          uint32_t cp = hex4();
          if (cp >= 0xD800 && cp < 0xDC00) {
            if (e - p < 6 || p[0] != '\\' || p[1] != 'u') fail("lone surrogate");
            p += 2;
            const uint32_t lo = hex4();
            if (lo < 0xDC00 || lo >= 0xE000) fail("bad surrogate pair");
            cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
          } else if (cp >= 0xDC00 && cp < 0xE000) {
            fail("lone surrogate");
          }
          put_utf8(o, cp);
          break;
        }
        default: fail("bad escape");
      }
    }
    return o;
  }
  JVal val(int depth = 0) {
    if (depth > 64) fail("nesting too deep");
    ws();
    if (p >= e) fail("unexpected end");
    JVal v;
    if (*p == '{') {
      v.t = JVal::Obj;
      ++p;
      ws();
      if (p < e && *p == '}') {
        ++p;
        return v;
      }
      while (true) {
        ws();
        std::string k = str();
        ws();
        if (p >= e || *p != ':') fail("expected ':'");
        ++p;
        v.o.emplace_back(std::move(k), val(depth + 1));
        ws();
        if (p < e && *p == ',') {
          ++p;
          continue;
        }
        if (p < e && *p == '}') {
          ++p;
          return v;
        }
        fail("expected ',' or '}'");
      }
    }
    if (*p == '[') {
      v.t = JVal::Arr;
      ++p;
      ws();
      if (p < e && *p == ']') {
        ++p;
        return v;
      }
      while (true) {
        v.a.push_back(val(depth + 1));
        ws();
        if (p < e && *p == ',') {
          ++p;
          continue;
        }
        if (p < e && *p == ']') {
          ++p;
          return v;
        }
        fail("expected ',' or ']'");
      }
    }
    if (*p == '"') {
      v.t = JVal::Str;
      v.s = str();
      return v;
    }
    if (e - p >= 4 && std::strncmp(p, "null", 4) == 0) {
      p += 4;
      return v;
    }
    if (e - p >= 4 && std::strncmp(p, "true", 4) == 0) {
      p += 4;
      v.t = JVal::Bool;
      v.b = true;
      return v;
    }
    if (e - p >= 5 && std::strncmp(p, "false", 5) == 0) {
      p += 5;
      v.t = JVal::Bool;
      return v;
    }
    // number
    const char *q = p;
    if (q < e && *q == '-') ++q;
    const char *digits = q;
    while (q < e && *q >= '0' && *q <= '9') ++q;
    if (q == digits) fail("unexpected character");
    bool integral = true;
    if (q < e && *q == '.') {
      integral = false;
      ++q;
      while (q < e && *q >= '0' && *q <= '9') ++q;
    }
    if (q < e && (*q == 'e' || *q == 'E')) {
      integral = false;
      ++q;
      if (q < e && (*q == '+' || *q == '-')) ++q;
      while (q < e && *q >= '0' && *q <= '9') ++q;
    }
    v.t = JVal::Num;
    const std::string txt(p, q);
    v.d = std::strtod(txt.c_str(), nullptr);
    if (integral && txt[0] != '-' && txt.size() <= 20) {
      uint64_t u = 0;
      bool ok = true;
      for (char c : txt) {
        const uint64_t nx = u * 10 + (uint64_t)(c - '0');
        if (nx / 10 != u) ok = false;
        u = nx;
      }
      v.is_uint = ok;
      v.u = u;
    }
    p = q;
    return v;
  }
};

uint64_t juint(const JVal *v, const char *field) {
  if (!v || v->t != JVal::Num || !v->is_uint)
    throw std::runtime_error(std::string("Invalid manifest JSON: field '") + field + "' is not an unsigned integer");
  return v->u;
}
std::string jstr(const JVal *v, const char *field) {
  if (!v || v->t != JVal::Str)
    throw std::runtime_error(std::string("Invalid manifest JSON: field '") + field + "' is not a string");
  return v->s;
}
}  // namespace

// ---------------------------------------------------------------------------
// writer (writer.rs:75-147, lib.rs:54-64)
// ---------------------------------------------------------------------------
void Writer::push(const std::string &name, const std::string &kind, uint64_t count, const void *data, size_t bytes) {
  Section s;
  s.name = name;
  s.kind = kind;
  s.count = count;
  s.offset = offset_;
  s.has_crc = true;
  s.crc = crc32((const uint8_t *)data, bytes);
  const Zstd *z = level > 0 ? zstd() : nullptr;
  if (level > 0 && !z) throw std::runtime_error("zstd compression requested but libzstd.so.1 is not available");
  Part part;
  part.p = (const uint8_t *)data;
  part.n = bytes;
  s.size = bytes;
  if (z) {
    std::vector<uint8_t> c(z->bound(bytes));
    const size_t r = z->compress(c.data(), c.size(), data, bytes, level);
    if (!z->is_error(r)) {  // the reference stores a section as is when compression fails
      c.resize(r);
      part.own = std::move(c);
      part.p = nullptr;
      part.n = r;
      s.size = r;
      s.compression = "zstd";
      s.has_usize = true;
      s.usize = bytes;
    }
  }
  offset_ += s.size;
  parts_.push_back(std::move(part));
  m.sections.push_back(s);
}

std::vector<uint8_t> Writer::head() const {
  const std::string h = manifest_json(m);
  std::vector<uint8_t> out;
  out.reserve(13 + h.size());
  out.insert(out.end(), {'T', 'A', 'A', 'S', '2'});
  const uint64_t n = h.size();
  for (int k = 0; k < 8; ++k) out.push_back((uint8_t)(n >> (8 * k)));
  out.insert(out.end(), h.begin(), h.end());
  return out;
}

std::vector<uint8_t> Writer::to_bytes() const {
  std::vector<uint8_t> out = head();
  for (const Part &p : parts_) {
    const uint8_t *d = p.own.empty() ? p.p : p.own.data();
    if (p.n) out.insert(out.end(), d, d + p.n);
  }
  return out;
}

void Writer::write(const std::string &path) const {
  const std::vector<uint8_t> h = head();
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("write " + path + ": cannot open");
  bool ok = std::fwrite(h.data(), 1, h.size(), f) == h.size();
  for (const Part &p : parts_) {
    const uint8_t *d = p.own.empty() ? p.p : p.own.data();
    ok = ok && (p.n == 0 || std::fwrite(d, 1, p.n, f) == p.n);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw std::runtime_error("write " + path + ": short write");
}

// ---------------------------------------------------------------------------
// reader (reader.rs:32-281)
// ---------------------------------------------------------------------------
void Reader::read_at(uint64_t off, void *dst, uint64_t n) const {
  if (n == 0) return;
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("Cannot open file: " + path);
  const bool ok = std::fseek(f, (long)off, SEEK_SET) == 0 && std::fread(dst, 1, (size_t)n, f) == (size_t)n;
  std::fclose(f);
  if (!ok) throw std::runtime_error("Cannot read file: " + path);
}

void Reader::open(const std::string &p) {
  path = p;
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) throw std::runtime_error("Cannot open file: " + path);
  bool ok = std::fseek(f, 0, SEEK_END) == 0;
  const long sz = ok ? std::ftell(f) : -1;
  std::fclose(f);
  if (!ok || sz < 0) throw std::runtime_error("Cannot read file: " + path);
  file_size = (uint64_t)sz;
  if (file_size < 13) throw std::runtime_error("File too short");
  uint8_t pre[13];
  read_at(0, pre, 13);
  if (std::memcmp(pre, "TAAS2", 5) != 0) {
    if (std::memcmp(pre, "TAAS1", 5) == 0)
      throw std::runtime_error("TAAS1 (the pre-v2 format) is not read here: migrate it to TAAS2 first");
    throw std::runtime_error("Invalid magic: expected TAAS2");
  }
  uint64_t hl = 0;
  for (int k = 0; k < 8; ++k) hl |= (uint64_t)pre[5 + k] << (8 * k);
  if (hl > file_size - 13) throw std::runtime_error("Header truncated");
  std::vector<char> hb((size_t)hl);
  read_at(13, hb.data(), hl);
  JParser jp{hb.data(), hb.data() + hb.size()};
  const JVal root = jp.val();
  jp.ws();
  if (jp.p != jp.e) throw std::runtime_error("Invalid manifest JSON: trailing characters");
  if (root.t != JVal::Obj) throw std::runtime_error("Invalid manifest JSON: not an object");
  m = Manifest{};
  m.version = jstr(root.get("version"), "version");
  m.created = jstr(root.get("created"), "created");
  const JVal *g = root.get("game");
  if (g && g->t != JVal::Null) {
    m.has_game = true;
    m.game = jstr(g, "game");
  }
  const JVal *secs = root.get("sections");
  if (!secs || secs->t != JVal::Arr) throw std::runtime_error("Invalid manifest JSON: no sections array");
  for (const JVal &sv : secs->a) {
    if (sv.t != JVal::Obj) throw std::runtime_error("Invalid manifest JSON: a section is not an object");
    Section s;
    s.name = jstr(sv.get("name"), "name");
    s.kind = jstr(sv.get("kind"), "kind");
    s.count = juint(sv.get("count"), "count");
    s.offset = juint(sv.get("offset"), "offset");
    s.size = juint(sv.get("size"), "size");
    const JVal *c = sv.get("crc32");
    if (c && c->t != JVal::Null) {
      const uint64_t v = juint(c, "crc32");
      if (v > 0xFFFFFFFFull) throw std::runtime_error("Invalid manifest JSON: crc32 out of range");
      s.has_crc = true;
      s.crc = (uint32_t)v;
    }
    const JVal *cm = sv.get("compression");
    if (cm && cm->t != JVal::Null) s.compression = jstr(cm, "compression");
    const JVal *us = sv.get("uncompressed_size");
    if (us && us->t != JVal::Null) {
      s.has_usize = true;
      s.usize = juint(us, "uncompressed_size");
    }
    m.sections.push_back(s);
  }
  const JVal *md = root.get("metadata");
  if (md && md->t == JVal::Obj)
    for (auto &kv : md->o) m.metadata[kv.first] = jstr(&kv.second, "metadata value");
  data_offset = 13 + hl;
  const uint64_t avail = file_size - data_offset;
  for (const Section &s : m.sections)
    if (s.offset > avail || s.size > avail - s.offset)
      throw std::runtime_error("Section '" + s.name + "' (offset=" + std::to_string(s.offset) + ", size=" +
                               std::to_string(s.size) + ") exceeds data (len=" + std::to_string(avail) + ")");
}

const Section *Reader::find(const std::string &name) const {
  for (const Section &s : m.sections)
    if (s.name == name) return &s;
  return nullptr;
}

uint64_t Reader::plain_size(const Section &s) const {
  if (s.compression.empty()) return s.size;
  if (s.has_usize) return s.usize;
  const Zstd *z = zstd();
  if (!z) throw std::runtime_error("Section '" + s.name + "' zstd decompression failed: libzstd.so.1 is not available");
  std::vector<uint8_t> head((size_t)std::min<uint64_t>(s.size, 18));
  read_at(data_offset + s.offset, head.data(), head.size());
  const unsigned long long n = z->content_size(head.data(), head.size());
  if (n >= (1ull << 62)) throw std::runtime_error("Section '" + s.name + "' zstd decompression failed: unknown size");
  return n;
}

uint64_t Reader::get_into(const std::string &name, const std::string &kind, void *dst, uint64_t cap) const {
  const Section *s = find(name);
  if (!s) throw std::runtime_error("Section '" + name + "' not found in manifest");
  if (s->kind != kind) throw std::runtime_error("Section '" + name + "' is not " + kind + ", got " + s->kind);
  if (!kind_known(kind)) throw std::runtime_error("Section '" + name + "' has unknown kind " + kind);
  if (!s->compression.empty() && s->compression != "zstd")
    throw std::runtime_error("Section '" + name + "' uses unknown compression " + s->compression);
  const uint64_t n = plain_size(*s);
  const size_t es = kind_size(kind);
  if (es && (s->count > UINT64_MAX / es || n != s->count * es))
    throw std::runtime_error("Section '" + name + "' " + kind + ": data len " + std::to_string(n) + " != count " +
                             std::to_string(s->count) + " * " + std::to_string(es));
  if (!dst) return n;
  if (cap < n) throw std::runtime_error("Section '" + name + "': output buffer too small");
  if (s->compression.empty()) {
    read_at(data_offset + s->offset, dst, n);
  } else {
    const Zstd *z = zstd();
    if (!z) throw std::runtime_error("Section '" + name + "' zstd decompression failed: libzstd.so.1 is not available");
    std::vector<uint8_t> src((size_t)s->size);
    read_at(data_offset + s->offset, src.data(), s->size);
    const size_t r = z->decompress(dst, (size_t)n, src.data(), src.size());
    if (z->is_error(r) || r != n) throw std::runtime_error("Section '" + name + "' zstd decompression failed");
  }
  if (s->has_crc) {
    const uint32_t c = crc32((const uint8_t *)dst, (size_t)n);
    if (c != s->crc) {
      char msg[160];
      std::snprintf(msg, sizeof msg, "CRC32 mismatch: expected %08x, got %08x", s->crc, c);
      throw std::runtime_error("Section '" + name + "' " + msg);
    }
  }
  return n;
}

std::vector<uint8_t> Reader::get(const std::string &name, const std::string &kind) const {
  std::vector<uint8_t> out((size_t)get_into(name, kind, nullptr, 0));
  get_into(name, kind, out.data(), out.size());
  return out;
}

// inspect.rs:5-64
static std::string human_size(uint64_t b) {
  char buf[64];
  if (b >= 1024 * 1024) std::snprintf(buf, sizeof buf, "%.1f MB", (double)b / (1024.0 * 1024.0));
  else if (b >= 1024) std::snprintf(buf, sizeof buf, "%.1f KB", (double)b / 1024.0);
  else std::snprintf(buf, sizeof buf, "%llu B", (unsigned long long)b);
  return buf;
}

std::string Reader::inspect() const {
  std::string o;
  char buf[512];
  o += "   Version: " + m.version + "\n";
  o += "   Created: " + m.created + "\n";
  if (m.has_game) o += "   Game:    " + m.game + "\n";
  o += "   Sections: " + std::to_string(m.sections.size()) + "\n\n";
  for (const Section &s : m.sections) {
    std::string sz = human_size(s.size);
    if (s.compression == "zstd") sz += " (uncompressed " + human_size(s.has_usize ? s.usize : 0) + ")";
    char crc[16];
    if (s.has_crc) std::snprintf(crc, sizeof crc, "%08x", s.crc);
    else std::snprintf(crc, sizeof crc, "-");
    std::snprintf(buf, sizeof buf, "   %-24s %-5s %10s  crc=%s  offset=%llu\n", s.name.c_str(), s.kind.c_str(),
                  sz.c_str(), crc, (unsigned long long)s.offset);
    o += buf;
    std::snprintf(buf, sizeof buf, "   %29s count=%llu\n", "", (unsigned long long)s.count);
    o += buf;
  }
  if (!m.metadata.empty()) {
    o += "\n   Metadata:\n";
    for (auto &kv : m.metadata) {
      std::snprintf(buf, sizeof buf, "      %-20s = ", kv.first.c_str());
      o += buf + kv.second + "\n";
    }
  }
  o += "\n   Total size: " + human_size(file_size);
  return o;
}

// lib.rs:68-78: the reference's clock fallback (year from days / 365.25,
// month and day fixed at 01-01, time of day from the clock)
std::string created_now() {
  const uint64_t secs = (uint64_t)std::time(nullptr);
  const uint64_t days = secs / 86400, tod = secs % 86400;
  const uint64_t year = 1970 + (uint64_t)((double)days / 365.25);
  char buf[64];
  std::snprintf(buf, sizeof buf, "%llu-01-01T%02llu:%02llu:%02lluZ", (unsigned long long)year,
                (unsigned long long)(tod / 3600), (unsigned long long)((tod % 3600) / 60),
                (unsigned long long)(tod % 60));
  return buf;
}

}  // namespace taas
}  // namespace sg
