// .taas v2 snapshot container (crates/SiMuse/crates/taas-format): the bytes
//   b"TAAS2" | header length u64 LE | UTF-8 JSON manifest | section payloads
// with a manifest {version, created, game?, sections: [{name, kind, count,
// offset, size, crc32?, compression?, uncompressed_size?}], metadata: {}}
// (types.rs:74-100), written compactly with the fields in that order and
// metadata keys sorted, as serde_json writes the reference's structs
// (lib.rs:54-64), so that the same snapshot gives the same bytes.  Each
// section's CRC32 (IEEE) is over its uncompressed bytes; a section may be
// zstd-compressed (writer.rs:79-101), through the system libzstd loaded at
// run time.  Host code only.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace sg {
namespace taas {

struct Section {
  std::string name, kind;
  uint64_t count = 0, offset = 0, size = 0;
  bool has_crc = false;
  uint32_t crc = 0;
  std::string compression;  // "" = stored as is
  bool has_usize = false;
  uint64_t usize = 0;
};

struct Manifest {
  std::string version = "2.0.0", created;
  bool has_game = false;
  std::string game;
  std::vector<Section> sections;
  std::map<std::string, std::string> metadata;
};

uint32_t crc32(const uint8_t *p, size_t n);  // threads over large buffers
size_t kind_size(const std::string &kind);    // element bytes of a numeric kind, 0 for str/json/blob
bool zstd_available();

class Writer {
 public:
  Manifest m;
  int level = 0;  // zstd level for the next sections, 0 = none
  // An uncompressed section's bytes are borrowed and must stay valid until
  // write(); a compressed section's bytes are kept here.
  void push(const std::string &name, const std::string &kind, uint64_t count, const void *data, size_t bytes);
  std::vector<uint8_t> head() const;      // magic, length, manifest
  std::vector<uint8_t> to_bytes() const;  // head + payload
  void write(const std::string &path) const;

 private:
  struct Part {
    const uint8_t *p = nullptr;
    size_t n = 0;
    std::vector<uint8_t> own;
  };
  std::vector<Part> parts_;
  uint64_t offset_ = 0;
};

class Reader {
 public:
  Manifest m;
  std::string path;
  uint64_t data_offset = 0, file_size = 0;
  // reads the magic, length and manifest only; throws std::runtime_error
  // with the reference's kind of message
  void open(const std::string &path);
  const Section *find(const std::string &name) const;
  // uncompressed bytes of a section of the given kind (kind, CRC and length
  // checked), read straight into dst (cap bytes); dst null: size only
  uint64_t get_into(const std::string &name, const std::string &kind, void *dst, uint64_t cap) const;
  std::vector<uint8_t> get(const std::string &name, const std::string &kind) const;
  std::string inspect() const;

 private:
  void read_at(uint64_t off, void *dst, uint64_t n) const;
  uint64_t plain_size(const Section &s) const;
};

std::string created_now();  // lib.rs:68-78 fallback timestamp

}  // namespace taas
}  // namespace sg
