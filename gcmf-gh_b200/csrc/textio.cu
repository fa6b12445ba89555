// textio.cu -- the GCMF text layer format, read in parallel on the host and written back.
//
// Format (dataConverter.py:95-111, read by ReadTextFormatPolygon2WithVector,
// SEQ_Overlay.h:285-390): the first line is a header and is skipped; then one polygon
// per line: "id minx miny maxx maxy x0 y0 x1 y1 ... x0 y0" (closing vertex repeated).
// Tokens are maximal runs of the characters 0-9 '.' '-' (getVertex, SEQ_Overlay.h:101-118;
// anything else separates, so exponent notation is not part of the format) and are
// converted with atof.  Reader rules restated from SEQ_Overlay.h:301-383:
//   * the first token is the polygon id; then coordinates are read as pairs until the
//     line ends; a final pair that parses as (0, 0) at the end of the line is dropped
//     (the empty tokens after the last vertex);
//   * the polygon's MBR is taken over every pair read, the two header pairs included;
//   * a polygon whose MBR has equal x (or y) extremes is skipped ("MBR Error!"), judged on
//     the 12-fraction-digit decimal keys of the extreme tokens (CoordToMBR, :69-97) and on
//     their FP64 values;
//   * the stored vertices are the pairs after the two header pairs, the closing one
//     included; vnum counts them and vps is their inclusive prefix sum.
// Deviations, all on inputs the reference cannot read: no 5,000,000-character line limit
// (MAX_BUFF), no 100,000-vertex polygon limit (MAX_VERTICES), and MBR extremes start at
// +/-infinity instead of +/-1,000,000, so coordinates beyond 1e6 are read correctly.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <vector>
#include "../../include/gcmfgh.h"

namespace {

inline bool tok_char(char c) { return c == '.' || c == '-' || (c >= '0' && c <= '9'); }

// CoordToMBR(token, 1): digits and sign of the token with at most 12 fraction digits,
// padded to 12, as an integer, plus 9e15.
long long decimal_key(const char* t, size_t n) {
  char buf[64];
  size_t i = 0;
  int frac = 0;
  bool dot = false;
  for (size_t k = 0; k < n && i < sizeof(buf) - 14; ++k) {
    if (t[k] != '.') {
      if (frac < 12) { buf[i++] = t[k]; if (dot) ++frac; }
      else break;
    } else {
      dot = true;
    }
  }
  for (; frac < 12 && i < sizeof(buf) - 1; ++frac) buf[i++] = '0';
  buf[i] = '\0';
  return atoll(buf) + 9000000000000000ll;
}

struct Parsed {
  std::vector<double> xy;
  std::vector<int32_t> vnum;
  std::vector<int64_t> id;
};

// One line; returns false when the polygon is skipped.
bool parse_line(const char* s, size_t len, Parsed& out) {
  size_t i = 0;
  auto next_token = [&](const char*& t, size_t& n) {
    while (i < len && !tok_char(s[i])) ++i;
    t = s + i;
    size_t st = i;
    while (i < len && tok_char(s[i])) ++i;
    n = i - st;
  };
  auto to_double = [](const char* t, size_t n) {
    char buf[128];
    if (n == 0) return 0.0;
    if (n >= sizeof(buf)) n = sizeof(buf) - 1;
    std::memcpy(buf, t, n);
    buf[n] = '\0';
    return atof(buf);
  };
  const char* t;
  size_t n;
  next_token(t, n);
  if (n == 0 && i >= len) return false;
  long long pid = (long long)to_double(t, n);
  std::vector<double> pts;
  double x1 = INFINITY, y1 = INFINITY, x2 = -INFINITY, y2 = -INFINITY;
  const char *tx1 = nullptr, *ty1 = nullptr, *tx2 = nullptr, *ty2 = nullptr;
  size_t nx1 = 0, ny1 = 0, nx2 = 0, ny2 = 0;
  for (;;) {
    const char *ta, *tb;
    size_t na, nb;
    next_token(ta, na);
    next_token(tb, nb);
    const bool at_end = i >= len;
    const double a = to_double(ta, na), b = to_double(tb, nb);
    if (at_end && a == 0.0 && b == 0.0) break;
    pts.push_back(a);
    pts.push_back(b);
    if (a < x1) { x1 = a; tx1 = ta; nx1 = na; }
    if (b < y1) { y1 = b; ty1 = tb; ny1 = nb; }
    if (a > x2) { x2 = a; tx2 = ta; nx2 = na; }
    if (b > y2) { y2 = b; ty2 = tb; ny2 = nb; }
    if (at_end) break;
  }
  const size_t npairs = pts.size() / 2;
  if (npairs < 2 || !tx1 || !ty1 || !tx2 || !ty2) return false;
  if (decimal_key(tx1, nx1) == decimal_key(tx2, nx2) || decimal_key(ty1, ny1) == decimal_key(ty2, ny2)) return false;
  if (x1 == x2 || y1 == y2) return false;
  out.xy.insert(out.xy.end(), pts.begin() + 4, pts.end());
  out.vnum.push_back((int32_t)(npairs - 2));
  out.id.push_back(pid);
  return true;
}

}  // namespace

extern "C" {

gcmfgh_status gcmfgh_read_text_layer(const char* path, int threads, gcmfgh_text_layer* out) {
  if (!path || !out) return GCMFGH_INVALID_ARGUMENT;
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return GCMFGH_INVALID_ARGUMENT;
  std::string buf;
  {
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (sz < 0) { std::fclose(f); return GCMFGH_INVALID_ARGUMENT; }
    buf.resize((size_t)sz);
    if (sz > 0 && std::fread(&buf[0], 1, (size_t)sz, f) != (size_t)sz) { std::fclose(f); return GCMFGH_INVALID_ARGUMENT; }
    std::fclose(f);
  }
  // line starts; the first line is the header
  std::vector<size_t> starts;
  size_t p = buf.find('\n');
  while (p != std::string::npos && p + 1 < buf.size()) {
    starts.push_back(p + 1);
    p = buf.find('\n', p + 1);
  }
  const size_t nl = starts.size();
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  threads = (int)std::max<size_t>(1, std::min<size_t>((size_t)threads, std::max<size_t>(1, nl / 64)));
  std::vector<Parsed> parts(threads);
  auto work = [&](int t) {
    size_t a = nl * t / threads, b = nl * (t + 1) / threads;
    for (size_t l = a; l < b; ++l) {
      size_t s0 = starts[l];
      size_t e = (l + 1 < nl) ? starts[l + 1] : buf.size();
      parse_line(buf.data() + s0, e - s0, parts[t]);
    }
  };
  if (threads == 1) work(0);
  else {
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  int64_t np = 0, nv = 0;
  for (auto& pt : parts) { np += (int64_t)pt.vnum.size(); nv += (int64_t)pt.xy.size() / 2; }
  out->coords = static_cast<double*>(std::malloc(sizeof(double) * 2 * std::max<int64_t>(nv, 1)));
  out->vnum = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * std::max<int64_t>(np, 1)));
  out->vps = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * std::max<int64_t>(np, 1)));
  out->ids = static_cast<int64_t*>(std::malloc(sizeof(int64_t) * std::max<int64_t>(np, 1)));
  if (!out->coords || !out->vnum || !out->vps || !out->ids) {
    gcmfgh_free_text_layer(out);
    return GCMFGH_OUT_OF_MEMORY;
  }
  int64_t ip = 0, iv = 0;
  for (auto& pt : parts) {
    std::copy(pt.xy.begin(), pt.xy.end(), out->coords + 2 * iv);
    for (size_t k = 0; k < pt.vnum.size(); ++k) {
      iv += pt.vnum[k];
      out->vnum[ip] = pt.vnum[k];
      out->vps[ip] = iv;
      out->ids[ip] = pt.id[k];
      ++ip;
    }
  }
  out->n_polys = np;
  out->n_vertices = nv;
  return GCMFGH_OK;
}

void gcmfgh_free_text_layer(gcmfgh_text_layer* L) {
  if (!L) return;
  std::free(L->coords);
  std::free(L->vnum);
  std::free(L->vps);
  std::free(L->ids);
  std::memset(L, 0, sizeof(*L));
}

// fixed-point text with 17 significant digits, so that atof returns the same double
static int fmt_coord(char* b, size_t cap, double v) {
  int e = (v == 0.0) ? 0 : (int)std::floor(std::log10(std::fabs(v)));
  int prec = std::min(std::max(16 - e, 1), 340);
  return std::snprintf(b, cap, "%.*f", prec, v);
}

gcmfgh_status gcmfgh_write_text_layer(const char* path, const gcmfgh_layer* L) {
  if (!path || !L || L->n_polys < 0 || (L->n_polys > 0 && (!L->coords || !L->vnum || !L->vps)))
    return GCMFGH_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "wb");
  if (!f) return GCMFGH_INVALID_ARGUMENT;
  std::fprintf(f, "%lld polygons\n", (long long)L->n_polys);
  char b[400];
  std::string line;
  for (int64_t i = 0; i < L->n_polys; ++i) {
    const int64_t e = L->vps[i], s = e - L->vnum[i];
    double x1 = INFINITY, y1 = INFINITY, x2 = -INFINITY, y2 = -INFINITY;
    for (int64_t k = s; k < e; ++k) {
      x1 = std::min(x1, L->coords[2 * k]); x2 = std::max(x2, L->coords[2 * k]);
      y1 = std::min(y1, L->coords[2 * k + 1]); y2 = std::max(y2, L->coords[2 * k + 1]);
    }
    line = std::to_string((long long)i);
    for (double v : {x1, y1, x2, y2}) { fmt_coord(b, sizeof(b), v); line += ' '; line += b; }
    for (int64_t k = s; k < e; ++k)
      for (int c = 0; c < 2; ++c) { fmt_coord(b, sizeof(b), L->coords[2 * k + c]); line += ' '; line += b; }
    line += " \n";
    std::fwrite(line.data(), 1, line.size(), f);
  }
  return std::fclose(f) == 0 ? GCMFGH_OK : GCMFGH_INVALID_ARGUMENT;
}

}  // extern "C"
