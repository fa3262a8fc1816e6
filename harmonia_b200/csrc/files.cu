// Reference dataset files and tree snapshots (host code).
//
// The reference reads its datasets as text, one signed decimal key per line
// (open-harmonia/src/main.cpp:50-67 for the insert file, the search loops of
// open-harmonia/src/full-multi-prefix-sort-8thread.cu for the query file, two
// lines per range in open-harmonia/src/range.cu:349-355), each line with
// sscanf("%lld").  The readers here accept the same lines: leading blanks are
// skipped, an optional sign and decimal digits are read, anything after the
// number is ignored.  Where sscanf would leave the key undefined (a line with
// no number) or saturate (a number outside int64), they return HM_EIO
// instead; blank lines are skipped.
//
// A snapshot is the tree's sorted contents and configuration in one binary
// file: header, n keys, n values, then a 64-bit checksum of the keys and
// values.  Loading it is a bulk load, so a tree written after upsert epochs
// comes back with the same contents (the shape is the bulk loader's).
#include "hm_internal.cuh"

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace hm {

namespace {

constexpr size_t kChunkBytes = 1 << 22;

struct FileCloser {
  void operator()(FILE *f) const {
    if (f) fclose(f);
  }
};
using File = std::unique_ptr<FILE, FileCloser>;

// Parses one line; returns 1 for a number, 0 for a blank line, -1 otherwise.
int parse_line(const char *p, const char *e, int64_t *out) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) p++;
  if (p == e) return 0;
  bool neg = false;
  if (*p == '+' || *p == '-') {
    neg = *p == '-';
    p++;
  }
  if (p == e || *p < '0' || *p > '9') return -1;
  uint64_t mag = 0;
  const uint64_t limit = neg ? (uint64_t)INT64_MAX + 1 : (uint64_t)INT64_MAX;
  for (; p < e && *p >= '0' && *p <= '9'; p++) {
    const uint64_t d = (uint64_t)(*p - '0');
    if (mag > (limit - d) / 10) return -1;  // outside int64
    mag = mag * 10 + d;
  }
  *out = neg ? (int64_t)(0 - mag) : (int64_t)mag;
  return 1;
}

// Calls fn(value) for every number line of the file, in order.
template <typename Fn>
int for_each_number(const char *path, Fn fn) {
  if (!path) return HM_EINVAL;
  File f(fopen(path, "rb"));
  if (!f) return HM_EIO;
  std::vector<char> buf(kChunkBytes);
  std::string carry;  // a line split across two reads
  for (;;) {
    const size_t got = fread(buf.data(), 1, buf.size(), f.get());
    if (got == 0) break;
    const char *p = buf.data(), *end = p + got;
    while (p < end) {
      const char *nl = static_cast<const char *>(memchr(p, '\n', (size_t)(end - p)));
      if (!nl) {
        carry.append(p, end);
        break;
      }
      int64_t v = 0;
      int r;
      if (!carry.empty()) {
        carry.append(p, nl);
        r = parse_line(carry.data(), carry.data() + carry.size(), &v);
        carry.clear();
      } else {
        r = parse_line(p, nl, &v);
      }
      if (r < 0) return HM_EIO;
      if (r > 0) fn(v);
      p = nl + 1;
    }
  }
  if (ferror(f.get())) return HM_EIO;
  if (!carry.empty()) {  // last line without a newline
    int64_t v = 0;
    const int r = parse_line(carry.data(), carry.data() + carry.size(), &v);
    if (r < 0) return HM_EIO;
    if (r > 0) fn(v);
  }
  return HM_OK;
}

// Checksum of the snapshot body: FNV-1a over 64-bit words.
uint64_t checksum(const int64_t *a, size_t n, uint64_t h) {
  for (size_t i = 0; i < n; i++) h = (h ^ (uint64_t)a[i]) * 0x100000001b3ull;
  return h;
}

constexpr char kMagic[8] = {'H', 'M', 'B', 'T', 'S', 'N', 'P', '1'};
constexpr uint32_t kVersion = 1;

struct SnapHeader {
  char magic[8];
  uint32_t version;
  uint32_t header_bytes;
  int32_t cfg[10];  // hm_config in declaration order
  int64_t n;
};

void cfg_to_words(const hm_config &c, int32_t *w) {
  const int v[10] = {c.fanout, c.leaf_cap, c.inner_fill, c.leaf_fill, c.group_width,
                     c.queries_per_group, c.sort_bits, c.smem_bytes, c.cache_hints, c.join};
  for (int i = 0; i < 10; i++) w[i] = v[i];
}

hm_config cfg_from_words(const int32_t *w) {
  hm_config c;
  c.fanout = w[0];
  c.leaf_cap = w[1];
  c.inner_fill = w[2];
  c.leaf_fill = w[3];
  c.group_width = w[4];
  c.queries_per_group = w[5];
  c.sort_bits = w[6];
  c.smem_bytes = w[7];
  c.cache_hints = w[8];
  c.join = w[9];
  return c;
}

bool write_all(FILE *f, const void *p, size_t bytes) { return fwrite(p, 1, bytes, f) == bytes; }
bool read_all(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes; }

}  // namespace

}  // namespace hm

using namespace hm;

extern "C" {

int hm_read_keys(const char *path, int64_t *keys, size_t cap, size_t *n) {
  if (!n) return HM_EINVAL;
  size_t count = 0;
  int rc = for_each_number(path, [&](int64_t v) {
    if (keys && count < cap) keys[count] = v;
    count++;
  });
  *n = count;
  if (rc) return rc;
  return keys && count > cap ? HM_ECAPACITY : HM_OK;
}

int hm_read_ranges(const char *path, int64_t *start, int64_t *end, size_t cap, size_t *n) {
  if (!n || (start == nullptr) != (end == nullptr)) return HM_EINVAL;
  size_t lines = 0;
  int rc = for_each_number(path, [&](int64_t v) {
    const size_t i = lines / 2;
    if (start && i < cap) (lines % 2 == 0 ? start : end)[i] = v;
    lines++;
  });
  *n = lines / 2;
  if (rc) return rc;
  if (lines % 2) return HM_EIO;  // a start without its end
  return start && *n > cap ? HM_ECAPACITY : HM_OK;
}

int hm_write_keys(const char *path, const int64_t *keys, size_t n) {
  if (!path || (n > 0 && !keys)) return HM_EINVAL;
  File f(fopen(path, "wb"));
  if (!f) return HM_EIO;
  std::vector<char> buf;
  buf.reserve(kChunkBytes + 32);
  for (size_t i = 0; i < n; i++) {
    char tmp[24];
    uint64_t mag = keys[i] < 0 ? 0 - (uint64_t)keys[i] : (uint64_t)keys[i];
    int l = 0;
    do {
      tmp[l++] = (char)('0' + mag % 10);
      mag /= 10;
    } while (mag);
    if (keys[i] < 0) buf.push_back('-');
    while (l) buf.push_back(tmp[--l]);
    buf.push_back('\n');
    if (buf.size() >= kChunkBytes) {
      if (!write_all(f.get(), buf.data(), buf.size())) return HM_EIO;
      buf.clear();
    }
  }
  if (!buf.empty() && !write_all(f.get(), buf.data(), buf.size())) return HM_EIO;
  return fflush(f.get()) == 0 ? HM_OK : HM_EIO;
}

int hm_snapshot_save(hm_tree *t, const char *path) {
  if (!t || !path) return HM_EINVAL;
  hm_tree_info info;
  int rc = hm_tree_get_info(t, &info);
  if (rc) return rc;
  const size_t n = (size_t)info.n_keys;
  std::vector<int64_t> k(n), v(n);
  size_t got = 0;
  rc = hm_export(t, k.data(), v.data(), n, &got);
  if (rc) return rc;
  SnapHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kMagic, sizeof(kMagic));
  h.version = kVersion;
  h.header_bytes = sizeof(SnapHeader);
  hm_config c;
  rc = hm_get_config(t, &c);
  if (rc) return rc;
  cfg_to_words(c, h.cfg);
  h.n = (int64_t)n;
  const uint64_t sum = checksum(v.data(), n, checksum(k.data(), n, 0xcbf29ce484222325ull));
  File f(fopen(path, "wb"));
  if (!f) return HM_EIO;
  if (!write_all(f.get(), &h, sizeof(h)) || !write_all(f.get(), k.data(), 8 * n) ||
      !write_all(f.get(), v.data(), 8 * n) || !write_all(f.get(), &sum, sizeof(sum)))
    return HM_EIO;
  return fflush(f.get()) == 0 ? HM_OK : HM_EIO;
}

int hm_snapshot_load(const char *path, const hm_config *cfg, hm_tree **out) {
  if (!path || !out) return HM_EINVAL;
  *out = nullptr;
  File f(fopen(path, "rb"));
  if (!f) return HM_EIO;
  SnapHeader h;
  if (!read_all(f.get(), &h, sizeof(h))) return HM_EIO;
  if (memcmp(h.magic, kMagic, sizeof(kMagic)) != 0 || h.version != kVersion ||
      h.header_bytes != sizeof(SnapHeader) || h.n < 0)
    return HM_EIO;
  // the file must hold exactly the header, 2n words and the checksum
  if (fseek(f.get(), 0, SEEK_END) != 0) return HM_EIO;
  const long size = ftell(f.get());
  if (size < 0 || (uint64_t)size != sizeof(SnapHeader) + 16ull * (uint64_t)h.n + 8ull) return HM_EIO;
  if (fseek(f.get(), (long)sizeof(SnapHeader), SEEK_SET) != 0) return HM_EIO;
  const size_t n = (size_t)h.n;
  std::vector<int64_t> k(n), v(n);
  uint64_t sum = 0;
  if (!read_all(f.get(), k.data(), 8 * n) || !read_all(f.get(), v.data(), 8 * n) ||
      !read_all(f.get(), &sum, sizeof(sum)))
    return HM_EIO;
  if (checksum(v.data(), n, checksum(k.data(), n, 0xcbf29ce484222325ull)) != sum) return HM_EIO;
  const hm_config saved = cfg_from_words(h.cfg);
  return hm_bulk_load(k.data(), v.data(), n, cfg ? cfg : &saved, out);
}

}  // extern "C"
