// Readers and writers of the reference's text input formats (host code).
//
//   Rect file (data/Rect1024.txt, read by BotomUp-rtree.cu:669-698 and
//   TopDown-rtree.cu:487-497): the record count, then per record
//   "x1 x2", "y1 y2" (integers) and an integer key.
//   Polygon file (the base and overlay files of readData,
//   vector_map_overlay_gpc_kernel.cu:752-888): the polygon count, then per
//   polygon its vertex count, its hole flag, its bounding box as four
//   doubles (x1 y1 x2 y2: readData tracks the minimum of the first as x and
//   of the second as y, GPC:808-813) and its vertices as "x y" pairs.
//   readData also quantises the box as (int)(v * 100000) (GPC:805-808).
//
// Whitespace between tokens is free, as for fscanf.  Numbers are parsed with
// strtoll / strtod (correctly rounded, like glibc's scanf) from a buffered
// stream, so files larger than memory are read in one pass.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

#include "prt_internal.cuh"

namespace prt {
namespace {

class TokenReader {
 public:
  explicit TokenReader(const char *path) : f_(fopen(path, "rb")), buf_(1 << 24) {}
  ~TokenReader() {
    if (f_) fclose(f_);
  }
  bool ok() const { return f_ != nullptr; }

  // Next whitespace-separated token into tok (NUL-terminated); false at EOF.
  bool next(char *tok, size_t cap) {
    int c;
    do {
      c = get();
    } while (c != EOF && isspace(c));
    if (c == EOF) return false;
    size_t k = 0;
    while (c != EOF && !isspace(c)) {
      if (k + 1 < cap) tok[k++] = (char)c;
      c = get();
    }
    tok[k] = '\0';
    return true;
  }

 private:
  int get() {
    if (pos_ == len_) {
      len_ = f_ ? fread(buf_.data(), 1, buf_.size(), f_) : 0;
      pos_ = 0;
      if (len_ == 0) return EOF;
    }
    return (unsigned char)buf_[pos_++];
  }
  FILE *f_;
  std::vector<char> buf_;
  size_t pos_ = 0, len_ = 0;
};

bool parse_i64(TokenReader &r, int64_t *v) {
  char t[64];
  if (!r.next(t, sizeof t)) return false;
  char *end = nullptr;
  errno = 0;
  long long x = strtoll(t, &end, 10);
  if (end == t || *end != '\0' || errno) return false;
  *v = x;
  return true;
}

bool parse_f64(TokenReader &r, double *v) {
  char t[128];
  if (!r.next(t, sizeof t)) return false;
  char *end = nullptr;
  double x = strtod(t, &end);
  if (end == t || *end != '\0') return false;
  *v = x;
  return true;
}

// readData's quantisation: (int)(v * 100000), truncation toward zero.
int32_t quantise(double v) {
  const double q = v * 100000.0;
  if (!(q > -2147483649.0 && q < 2147483648.0)) return q > 0 ? std::numeric_limits<int32_t>::max()
                                                               : std::numeric_limits<int32_t>::min();
  return (int32_t)q;
}

}  // namespace
}  // namespace prt

using namespace prt;

extern "C" {

int prt_rect_file_count(const char *path, int64_t *n) {
  PRT_CHECK(path && n, PRT_ERR_INVALID, "NULL argument");
  TokenReader r(path);
  PRT_CHECK(r.ok(), PRT_ERR_INVALID, "%s: cannot open", path);
  PRT_CHECK(parse_i64(r, n) && *n >= 0, PRT_ERR_INVALID, "%s: no record count", path);
  return PRT_OK;
}

int prt_read_rect_file(const char *path, int64_t *h_boxes, int32_t *h_keys, int64_t cap, int64_t *n_read) {
  PRT_CHECK(path && n_read, PRT_ERR_INVALID, "NULL argument");
  TokenReader r(path);
  PRT_CHECK(r.ok(), PRT_ERR_INVALID, "%s: cannot open", path);
  int64_t n = 0;
  PRT_CHECK(parse_i64(r, &n) && n >= 0, PRT_ERR_INVALID, "%s: no record count", path);
  *n_read = n;
  PRT_CHECK(n <= cap, PRT_ERR_CAPACITY, "%s: %lld records, room for %lld", path, (long long)n, (long long)cap);
  PRT_CHECK(n == 0 || h_boxes, PRT_ERR_INVALID, "NULL argument");
  for (int64_t i = 0; i < n; i++) {
    int64_t x1, x2, y1, y2, key;
    PRT_CHECK(parse_i64(r, &x1) && parse_i64(r, &x2) && parse_i64(r, &y1) && parse_i64(r, &y2) &&
                  parse_i64(r, &key),
              PRT_ERR_INVALID, "%s: record %lld is malformed", path, (long long)i);
    h_boxes[4 * i] = x1;
    h_boxes[4 * i + 1] = y1;
    h_boxes[4 * i + 2] = x2;
    h_boxes[4 * i + 3] = y2;
    if (h_keys) h_keys[i] = (int32_t)key;
  }
  return PRT_OK;
}

int prt_write_rect_file(const char *path, const int64_t *h_boxes, const int32_t *h_keys, int64_t n) {
  PRT_CHECK(path && (n == 0 || h_boxes) && n >= 0, PRT_ERR_INVALID, "bad argument");
  FILE *f = fopen(path, "w");
  PRT_CHECK(f, PRT_ERR_INVALID, "%s: cannot create", path);
  fprintf(f, "%lld\n", (long long)n);
  for (int64_t i = 0; i < n; i++) {
    const int64_t *b = h_boxes + 4 * i;
    fprintf(f, "%lld %lld\n%lld %lld\n%d\n", (long long)b[0], (long long)b[2], (long long)b[1], (long long)b[3],
            h_keys ? h_keys[i] : (int)i);
  }
  const bool ok = !ferror(f);
  fclose(f);
  PRT_CHECK(ok, PRT_ERR_INVALID, "%s: write failed", path);
  return PRT_OK;
}

int prt_polygon_file_size(const char *path, int64_t *n_poly, int64_t *n_vert) {
  PRT_CHECK(path && n_poly && n_vert, PRT_ERR_INVALID, "NULL argument");
  TokenReader r(path);
  PRT_CHECK(r.ok(), PRT_ERR_INVALID, "%s: cannot open", path);
  int64_t n = 0, total = 0;
  PRT_CHECK(parse_i64(r, &n) && n >= 0, PRT_ERR_INVALID, "%s: no polygon count", path);
  char t[128];
  for (int64_t i = 0; i < n; i++) {
    int64_t num = 0, hole = 0;
    PRT_CHECK(parse_i64(r, &num) && num >= 0 && parse_i64(r, &hole), PRT_ERR_INVALID,
              "%s: polygon %lld header is malformed", path, (long long)i);
    for (int64_t k = 0; k < 4 + 2 * num; k++)
      PRT_CHECK(r.next(t, sizeof t), PRT_ERR_INVALID, "%s: polygon %lld is truncated", path, (long long)i);
    total += num;
  }
  *n_poly = n;
  *n_vert = total;
  return PRT_OK;
}

int prt_read_polygon_file(const char *path, int32_t *h_num, int64_t *h_prefix, int32_t *h_hole, double *h_mbr,
                          int32_t *h_rect, double *h_vertex, int64_t poly_cap, int64_t vert_cap) {
  PRT_CHECK(path, PRT_ERR_INVALID, "NULL argument");
  TokenReader r(path);
  PRT_CHECK(r.ok(), PRT_ERR_INVALID, "%s: cannot open", path);
  int64_t n = 0;
  PRT_CHECK(parse_i64(r, &n) && n >= 0, PRT_ERR_INVALID, "%s: no polygon count", path);
  PRT_CHECK(n <= poly_cap, PRT_ERR_CAPACITY, "%s: %lld polygons, room for %lld", path, (long long)n,
            (long long)poly_cap);
  PRT_CHECK(n == 0 || (h_num && h_prefix && h_hole), PRT_ERR_INVALID, "NULL argument");
  int64_t v = 0;
  for (int64_t i = 0; i < n; i++) {
    int64_t num = 0, hole = 0;
    PRT_CHECK(parse_i64(r, &num) && num >= 0 && num < (1ll << 31) && parse_i64(r, &hole), PRT_ERR_INVALID,
              "%s: polygon %lld header is malformed", path, (long long)i);
    double m[4];
    for (int k = 0; k < 4; k++)
      PRT_CHECK(parse_f64(r, &m[k]), PRT_ERR_INVALID, "%s: polygon %lld box is malformed", path, (long long)i);
    h_num[i] = (int32_t)num;
    h_hole[i] = (int32_t)hole;
    h_prefix[i] = v;  // prefix[i] = prefix[i-1] + num[i-1] (GPC:797-802)
    for (int k = 0; k < 4; k++) {
      if (h_mbr) h_mbr[4 * i + k] = m[k];
      if (h_rect) h_rect[4 * i + k] = quantise(m[k]);
    }
    PRT_CHECK(v + num <= vert_cap, PRT_ERR_CAPACITY, "%s: more than %lld vertices", path, (long long)vert_cap);
    for (int64_t k = 0; k < num; k++) {
      double x, y;
      PRT_CHECK(parse_f64(r, &x) && parse_f64(r, &y), PRT_ERR_INVALID, "%s: polygon %lld vertex %lld is malformed",
                path, (long long)i, (long long)k);
      if (h_vertex) {
        h_vertex[2 * (v + k)] = x;
        h_vertex[2 * (v + k) + 1] = y;
      }
    }
    v += num;
  }
  return PRT_OK;
}

int prt_write_polygon_file(const char *path, const int32_t *h_num, const int32_t *h_hole, const double *h_vertex,
                           int64_t n_poly) {
  PRT_CHECK(path && n_poly >= 0 && (n_poly == 0 || (h_num && h_vertex)), PRT_ERR_INVALID, "bad argument");
  FILE *f = fopen(path, "w");
  PRT_CHECK(f, PRT_ERR_INVALID, "%s: cannot create", path);
  fprintf(f, "%lld\n", (long long)n_poly);
  int64_t v = 0;
  for (int64_t i = 0; i < n_poly; i++) {
    const int num = h_num[i];
    double x1 = 0, y1 = 0, x2 = 0, y2 = 0;
    for (int k = 0; k < num; k++) {
      const double x = h_vertex[2 * (v + k)], y = h_vertex[2 * (v + k) + 1];
      if (k == 0 || x < x1) x1 = x;
      if (k == 0 || y < y1) y1 = y;
      if (k == 0 || x > x2) x2 = x;
      if (k == 0 || y > y2) y2 = y;
    }
    // %.17g: every double reads back to the same value
    fprintf(f, "%d %d\n%.17g %.17g %.17g %.17g\n", num, h_hole ? h_hole[i] : 0, x1, y1, x2, y2);
    for (int k = 0; k < num; k++) fprintf(f, "%.17g %.17g\n", h_vertex[2 * (v + k)], h_vertex[2 * (v + k) + 1]);
    v += num;
  }
  const bool ok = !ferror(f);
  fclose(f);
  PRT_CHECK(ok, PRT_ERR_INVALID, "%s: write failed", path);
  return PRT_OK;
}

}  // extern "C"
