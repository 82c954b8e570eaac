// Host-side polyMesh reader/writer, geometry and synthetic channel meshes.
// Reader grammar and geometry follow apps/generic_simple_v1/src/main.cu:532-599.
#include "host_mesh.hpp"

#include <algorithm>
#include <cctype>
#include <climits>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <sys/stat.h>
#include <tuple>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace anb {
namespace {

inline Vec3 add3(const Vec3& a, const Vec3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline Vec3 sub3(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline Vec3 mul3(double s, const Vec3& a) { return {s * a[0], s * a[1], s * a[2]}; }
inline double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline Vec3 cross3(const Vec3& a, const Vec3& b) {
  return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
inline double norm3(const Vec3& a) { return std::sqrt(dot3(a, a)); }

std::string read_file(const std::string& fn) {
  std::ifstream in(fn, std::ios::binary);
  if (!in) throw std::runtime_error("Could not open " + fn);
  std::string s;
  in.seekg(0, std::ios::end);
  std::streamoff n = in.tellg();
  if (n > 0) {
    s.resize((size_t)n);
    in.seekg(0, std::ios::beg);
    in.read(&s[0], n);
  }
  return s;
}

// Removes /* */ blocks (an unterminated one stays) and // line comments, main.cu:533-537, in one
// linear pass each.  The reference erases the first "/*" ... "*/" block and searches the edited
// string again from its start, so a '/' just before an erased block and a '*' just after it form a
// new block start; the scan below reproduces that.
std::string strip_comments(std::string txt) {
  const size_t npos = std::string::npos;
  std::string s;
  size_t i = 0;
  const bool blocks = txt.find("/*") != npos;
  if (!blocks) s = std::move(txt);  // no block comment: nothing to erase
  else s.reserve(txt.size());
  while (blocks) {
    const size_t a = txt.find("/*", i);
    if (a == npos) {
      s.append(txt, i, npos);
      break;
    }
    const size_t b = txt.find("*/", a + 2);
    if (b == npos) {  // unterminated: the rest stays as it is
      s.append(txt, i, npos);
      break;
    }
    s.append(txt, i, a - i);
    i = b + 2;
    // a '/' left before the erased block and a '*' after it make the next block start
    bool stop = false;
    while (!s.empty() && s.back() == '/' && i < txt.size() && txt[i] == '*') {
      const size_t e = txt.find("*/", i + 1);
      if (e == npos) {  // unterminated: the reference stops erasing here, the rest stays
        s.append(txt, i, npos);
        stop = true;
        break;
      }
      s.pop_back();
      i = e + 2;
    }
    if (stop) break;
  }
  // line comments: each line keeps what precedes its first "//" and ends with '\n' (the
  // reference's getline loop); lines without "//" are copied in bulk up to the next occurrence
  std::string out;
  out.reserve(s.size() + 1);
  const size_t n = s.size();
  size_t a = 0;
  while (a < n) {
    const size_t c = s.find("//", a);
    if (c == npos) {
      out.append(s, a, npos);
      if (out.back() != '\n') out.push_back('\n');
      break;
    }
    out.append(s, a, c - a);
    out.push_back('\n');
    const size_t nl = s.find('\n', c);
    if (nl == npos) break;
    a = nl + 1;
  }
  return out;
}

// files (list bodies) larger than this are scanned and parsed by all host threads
constexpr size_t kParallelParseBytes = 1 << 20;

int parse_threads() {
#ifdef _OPENMP
  return std::max(1, omp_get_max_threads());
#else
  return 1;
#endif
}

// First "<digits> (" opens the top-level list; returns its inside (main.cu:538-546).
std::pair<size_t, size_t> main_list_range(const std::string& t) {
  size_t start = std::string::npos, open = std::string::npos;
  for (size_t i = 0; i < t.size(); ++i) {
    if (std::isdigit((unsigned char)t[i])) {
      size_t j = i;
      while (j < t.size() && std::isdigit((unsigned char)t[j])) ++j;
      while (j < t.size() && std::isspace((unsigned char)t[j])) ++j;
      if (j < t.size() && t[j] == '(') {
        start = i;
        open = j;
        break;
      }
    }
  }
  if (start == std::string::npos) throw std::runtime_error("Could not locate top-level OpenFOAM list");
  // the matching ')' is the first position where the running depth (1 after the opening '(')
  // returns to 0; large files are scanned in chunks: the net depth change and the lowest running
  // depth of each chunk in parallel, then the first chunk whose lowest depth reaches 0 is scanned
  // again from its starting depth for the exact position
  const size_t n = t.size();
  size_t close = std::string::npos;
  const int nT = parse_threads();
  size_t from = open;
  long long depth = 0;
  if (n - open > kParallelParseBytes && nT > 1) {
    const int nC = 4 * nT;
    const size_t len = n - open;
    std::vector<long long> net(nC, 0), low(nC, 0);
#pragma omp parallel for schedule(static) num_threads(nT)
    for (int k = 0; k < nC; ++k) {
      const size_t b = open + len * (size_t)k / nC, e = open + len * (size_t)(k + 1) / nC;
      long long d = 0, lo = LLONG_MAX;
      for (size_t i = b; i < e; ++i) {
        const char c = t[i];
        d += (c == '(') - (c == ')');
        lo = std::min(lo, d);
      }
      net[k] = d;
      low[k] = lo;
    }
    from = n;  // no chunk closes: nothing to scan, "Failed to match parentheses" below
    long long base = 0;
    for (int k = 0; k < nC; ++k) {
      if (low[k] != LLONG_MAX && base + low[k] <= 0) {
        from = open + len * (size_t)k / nC;
        depth = base;
        break;
      }
      base += net[k];
    }
  }
  for (size_t i = from; i < n; ++i) {
    if (t[i] == '(') ++depth;
    else if (t[i] == ')') {
      --depth;
      if (depth == 0) {
        close = i;
        break;
      }
    }
  }
  if (close == std::string::npos) throw std::runtime_error("Failed to match parentheses");
  return {open + 1, close};
}

// istream-like integer parse inside [p, e): skips whitespace, returns false if no integer.
inline bool parse_int(const char*& p, const char* e, int& v) {
  while (p < e && std::isspace((unsigned char)*p)) ++p;
  const char* q = p;
  bool neg = false;
  if (q < e && (*q == '-' || *q == '+')) {
    neg = (*q == '-');
    ++q;
  }
  if (q >= e || !std::isdigit((unsigned char)*q)) return false;
  long long acc = 0;
  while (q < e && std::isdigit((unsigned char)*q)) {
    acc = acc * 10 + (*q - '0');
    ++q;
  }
  v = (int)(neg ? -acc : acc);
  p = q;
  return true;
}

inline bool parse_double(const char*& p, const char* e, double& v) {
  while (p < e && std::isspace((unsigned char)*p)) ++p;
  if (p >= e) return false;
  char buf[64];
  size_t len = 0;
  while (p + len < e && len < 63 && !std::isspace((unsigned char)p[len]) && p[len] != ')') {
    buf[len] = p[len];
    ++len;
  }
  buf[len] = 0;
  char* end = nullptr;
  errno = 0;
  double d = std::strtod(buf, &end);
  if (end == buf) return false;
  v = d;
  p += (end - buf);
  return true;
}

// ---- parallel parse of well-formed list bodies ---------------------------------------------
// Large lists are cut into one chunk per thread and parsed concurrently under a strict grammar
// (every entry complete, every token fully consumed, nothing else but whitespace).  A body that
// passes the strict grammar everywhere is parsed by the serial readers below into exactly the
// same values (they use the same token parsers and see the same entries in the same order), so
// the result is identical; any deviation sends the whole file to the serial reader, whose
// behaviour on odd input (skipped garbage, missing or extra tokens) is the reference's.

// the C locale's isspace set: ' ', \t, \n, \v, \f, \r
inline bool is_ws(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }
inline void skip_ws(const char*& p, const char* e) {
  while (p < e && is_ws(*p)) ++p;
}
// parse_int for the strict paths (same result; the C locale's whitespace set inline)
inline bool parse_int_fast(const char*& p, const char* e, int& v) {
  while (p < e && is_ws(*p)) ++p;
  const char* q = p;
  bool neg = false;
  if (q < e && (*q == '-' || *q == '+')) {
    neg = (*q == '-');
    ++q;
  }
  if (q >= e || (unsigned)(*q - '0') > 9u) return false;
  long long acc = 0;
  while (q < e && (unsigned)(*q - '0') <= 9u) acc = acc * 10 + (*q++ - '0');
  v = (int)(neg ? -acc : acc);
  p = q;
  return true;
}

// the token just parsed ended at whitespace, ')' or the end
inline bool token_end(const char* p, const char* e) { return p >= e || is_ws(*p) || *p == ')'; }

// Chunk starts for nT threads: each cut lies just after a `sep` character (')' for lists of
// parenthesised entries) or on whitespace (sep == 0, lists of bare labels).
std::vector<const char*> chunk_cuts(const char* b, const char* e, int nT, char sep) {
  std::vector<const char*> cut{b};
  const size_t len = (size_t)(e - b);
  for (int k = 1; k < nT; ++k) {
    const char* q = std::max(cut.back(), b + len * (size_t)k / (size_t)nT);
    if (sep) {
      q = static_cast<const char*>(std::memchr(q, sep, (size_t)(e - q)));
      q = q ? q + 1 : e;
    } else {
      while (q < e && !is_ws(*q)) ++q;
    }
    cut.push_back(q);
  }
  cut.push_back(e);
  return cut;
}

// out = the chunks' vectors one after the other, copied in parallel
template <class T>
void concat_parallel(const std::vector<std::vector<T>>& part, std::vector<T>& out) {
  std::vector<size_t> at(part.size() + 1, 0);
  for (size_t k = 0; k < part.size(); ++k) at[k + 1] = at[k] + part[k].size();
  out.resize(at.back());
#pragma omp parallel for schedule(static, 1)
  for (int k = 0; k < (int)part.size(); ++k)
    if (!part[k].empty()) std::memcpy(out.data() + at[k], part[k].data(), part[k].size() * sizeof(T));
}

// points: "(x y z)" entries
bool parse_points_parallel(const char* b, const char* e, std::vector<Vec3>& out) {
  const int nT = parse_threads();
  if ((size_t)(e - b) < kParallelParseBytes || nT < 2) return false;
  const std::vector<const char*> cut = chunk_cuts(b, e, nT, ')');
  std::vector<std::vector<Vec3>> part(nT);
  std::vector<char> ok(nT, 1);
#pragma omp parallel for schedule(static, 1) num_threads(nT)
  for (int k = 0; k < nT; ++k) {
    const char* p = cut[k];
    const char* ce = cut[k + 1];
    auto& v = part[k];
    v.reserve((size_t)(ce - p) / 40 + 1);
    while (true) {
      skip_ws(p, ce);
      if (p >= ce) break;
      if (*p != '(') { ok[k] = 0; break; }
      ++p;
      Vec3 x{0.0, 0.0, 0.0};
      bool good = true;
      for (int q = 0; q < 3 && good; ++q) good = parse_double(p, ce, x[q]) && token_end(p, ce);
      skip_ws(p, ce);
      if (!good || p >= ce || *p != ')') { ok[k] = 0; break; }
      ++p;
      v.push_back(x);
    }
  }
  for (char c : ok)
    if (!c) return false;
  concat_parallel(part, out);
  return true;
}

// faces: "k(v0 ... vk-1)" entries
bool parse_faces_parallel(const char* b, const char* e, std::vector<int>& off, std::vector<int>& pts) {
  const int nT = parse_threads();
  if ((size_t)(e - b) < kParallelParseBytes || nT < 2) return false;
  const std::vector<const char*> cut = chunk_cuts(b, e, nT, ')');
  std::vector<std::vector<int>> cnt(nT), vals(nT);
  std::vector<char> ok(nT, 1);
#pragma omp parallel for schedule(static, 1) num_threads(nT)
  for (int k = 0; k < nT; ++k) {
    const char* p = cut[k];
    const char* ce = cut[k + 1];
    auto& c = cnt[k];
    auto& v = vals[k];
    c.reserve((size_t)(ce - p) / 20 + 1);
    v.reserve((size_t)(ce - p) / 5 + 1);
    while (true) {
      skip_ws(p, ce);
      if (p >= ce) break;
      if (!std::isdigit((unsigned char)*p)) { ok[k] = 0; break; }
      long long n = 0;
      while (p < ce && std::isdigit((unsigned char)*p) && n < (1LL << 40)) n = n * 10 + (*p++ - '0');
      skip_ws(p, ce);
      if (p >= ce || *p != '(' || n >= (1LL << 31)) { ok[k] = 0; break; }
      ++p;
      bool good = true;
      for (long long i = 0; i < n && good; ++i) {
        int x = 0;
        good = parse_int_fast(p, ce, x) && token_end(p, ce);
        v.push_back(x);
      }
      skip_ws(p, ce);
      if (!good || p >= ce || *p != ')') { ok[k] = 0; break; }
      ++p;
      c.push_back((int)n);
    }
  }
  for (char c : ok)
    if (!c) return false;
  size_t nf = 0, np = 0;
  for (int k = 0; k < nT; ++k) {
    nf += cnt[k].size();
    np += vals[k].size();
  }
  if (np >= (size_t)INT32_MAX) return false;
  concat_parallel(vals, pts);
  std::vector<int> sizes;
  concat_parallel(cnt, sizes);
  off.resize(nf + 1);
  off[0] = 0;
  for (size_t f = 0; f < nf; ++f) off[f + 1] = off[f] + sizes[f];
  return true;
}

// labels: whitespace-separated integers
bool parse_labels_parallel(const char* b, const char* e, std::vector<int>& out) {
  const int nT = parse_threads();
  if ((size_t)(e - b) < kParallelParseBytes || nT < 2) return false;
  const std::vector<const char*> cut = chunk_cuts(b, e, nT, 0);
  std::vector<std::vector<int>> part(nT);
  std::vector<char> ok(nT, 1);
#pragma omp parallel for schedule(static, 1) num_threads(nT)
  for (int k = 0; k < nT; ++k) {
    const char* p = cut[k];
    const char* ce = cut[k + 1];
    auto& v = part[k];
    v.reserve((size_t)(ce - p) / 6 + 1);
    while (true) {
      skip_ws(p, ce);
      if (p >= ce) break;
      int x = 0;
      if (!parse_int_fast(p, ce, x) || (p < ce && !is_ws(*p))) { ok[k] = 0; break; }
      v.push_back(x);
    }
  }
  for (char c : ok)
    if (!c) return false;
  concat_parallel(part, out);
  return true;
}

std::vector<Vec3> read_points(const std::string& fn) {
  std::string t = strip_comments(read_file(fn));
  auto r = main_list_range(t);
  {
    std::vector<Vec3> P;
    if (parse_points_parallel(t.data() + r.first, t.data() + r.second, P)) return P;
  }
  std::vector<Vec3> P;
  const char* base = t.data();
  size_t pos = r.first;
  while (true) {
    size_t a = t.find('(', pos);
    if (a == std::string::npos || a >= r.second) break;
    size_t b = t.find(')', a + 1);
    if (b == std::string::npos || b > r.second) break;
    const char* p = base + a + 1;
    const char* e = base + b;
    Vec3 x{0.0, 0.0, 0.0};
    for (int k = 0; k < 3; ++k)
      if (!parse_double(p, e, x[k])) break;
    P.push_back(x);
    pos = b + 1;
  }
  return P;
}

void read_faces(const std::string& fn, std::vector<int>& off, std::vector<int>& pts) {
  std::string t = strip_comments(read_file(fn));
  auto r = main_list_range(t);
  if (parse_faces_parallel(t.data() + r.first, t.data() + r.second, off, pts)) return;
  off.assign(1, 0);
  pts.clear();
  const char* base = t.data();
  size_t pos = r.first, end = r.second;
  while (pos < end) {
    while (pos < end && std::isspace((unsigned char)t[pos])) ++pos;
    if (pos >= end) break;
    if (!std::isdigit((unsigned char)t[pos])) {
      ++pos;
      continue;
    }
    size_t q = pos;
    long long k = 0;
    while (q < end && std::isdigit((unsigned char)t[q])) {
      k = k * 10 + (t[q] - '0');
      ++q;
    }
    while (q < end && std::isspace((unsigned char)t[q])) ++q;
    if (q >= end || t[q] != '(') throw std::runtime_error("Malformed faces list");
    size_t rr = t.find(')', q + 1);
    if (rr == std::string::npos || rr > end) throw std::runtime_error("Malformed faces list");
    const char* p = base + q + 1;
    const char* e = base + rr;
    bool ok = true;
    for (long long i = 0; i < k; ++i) {
      int v = 0;
      if (ok && !parse_int(p, e, v)) {
        ok = false;
        v = 0;
      }
      pts.push_back(ok ? v : 0);
    }
    off.push_back((int)pts.size());
    pos = rr + 1;
  }
}

std::vector<int> read_labels(const std::string& fn) {
  std::string t = strip_comments(read_file(fn));
  auto r = main_list_range(t);
  std::vector<int> v;
  if (parse_labels_parallel(t.data() + r.first, t.data() + r.second, v)) return v;
  const char* p = t.data() + r.first;
  const char* e = t.data() + r.second;
  int x;
  while (parse_int(p, e, x)) {
    v.push_back(x);
    if (p < e && !std::isspace((unsigned char)*p)) break;
  }
  return v;
}

std::vector<PatchInfo> read_boundary(const std::string& fn) {
  std::string t = strip_comments(read_file(fn));
  auto r = main_list_range(t);
  std::string inside = t.substr(r.first, r.second - r.first);
  std::vector<PatchInfo> out;
  size_t pos = 0;
  while (pos < inside.size()) {
    while (pos < inside.size() && std::isspace((unsigned char)inside[pos])) ++pos;
    if (pos >= inside.size()) break;
    if (!(std::isalpha((unsigned char)inside[pos]) || inside[pos] == '_')) {
      ++pos;
      continue;
    }
    size_t a = pos;
    while (pos < inside.size() && (std::isalnum((unsigned char)inside[pos]) || inside[pos] == '_')) ++pos;
    std::string name = inside.substr(a, pos - a);
    while (pos < inside.size() && std::isspace((unsigned char)inside[pos])) ++pos;
    if (pos >= inside.size() || inside[pos] != '{') continue;
    int depth = 1;
    size_t bodyStart = ++pos;
    while (pos < inside.size() && depth > 0) {
      if (inside[pos] == '{') ++depth;
      else if (inside[pos] == '}') --depth;
      ++pos;
    }
    std::string body = inside.substr(bodyStart, pos - bodyStart - 1);
    auto find_int = [&](const std::string& key) -> int {
      size_t k = body.find(key);
      if (k == std::string::npos) return 0;
      k += key.size();
      while (k < body.size() && !std::isdigit((unsigned char)body[k]) && body[k] != '-') ++k;
      size_t e = k;
      while (e < body.size() && (std::isdigit((unsigned char)body[e]) || body[e] == '-')) ++e;
      return std::atoi(body.substr(k, e - k).c_str());
    };
    auto find_word = [&](const std::string& key) -> std::string {
      size_t k = body.find(key);
      if (k == std::string::npos) return "";
      k += key.size();
      while (k < body.size() && std::isspace((unsigned char)body[k])) ++k;
      size_t e = k;
      while (e < body.size() && (std::isalnum((unsigned char)body[e]) || body[e] == '_')) ++e;
      return body.substr(k, e - k);
    };
    PatchInfo p;
    p.name = name;
    p.nFaces = find_int("nFaces");
    p.start = find_int("startFace");
    p.type = find_word("type");
    out.push_back(p);
  }
  return out;
}

void write_header(std::ostream& o, const char* cls, const char* obj, const std::string& note) {
  o << "/*--------------------------------*- C++ -*----------------------------------*\\\n"
       "  Written by anabasis_b200 (synthetic mesh)\n"
       "\\*---------------------------------------------------------------------------*/\n"
       "FoamFile\n{\n    format      ascii;\n    class       "
    << cls << ";\n";
  if (!note.empty()) o << "    note        \"" << note << "\";\n";
  o << "    location    \"constant/polyMesh\";\n    object      " << obj
    << ";\n}\n// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //\n\n";
}

void mkdir_p(const std::string& dir) {
  std::string cur;
  for (size_t i = 0; i <= dir.size(); ++i) {
    if (i == dir.size() || dir[i] == '/') {
      if (!cur.empty()) ::mkdir(cur.c_str(), 0755);
    }
    if (i < dir.size()) cur.push_back(dir[i]);
  }
}

}  // namespace

void finalize_topology(HostMesh& m) {
  m.nFaces = (int)m.faceOff.size() - 1;
  m.nInternalFaces = (int)m.neigh.size();
  if ((int)m.owner.size() < m.nFaces)
    throw std::runtime_error("owner list shorter than faces list");
  m.owner.resize(m.nFaces);
  m.nCells = 0;
  for (int v : m.owner) m.nCells = std::max(m.nCells, v + 1);
  for (int v : m.neigh) m.nCells = std::max(m.nCells, v + 1);
  m.bPatch.assign(m.nFaces, 0);
  for (size_t k = 0; k < m.patches.size(); ++k)
    for (int f = m.patches[k].start; f < m.patches[k].start + m.patches[k].nFaces; ++f)
      if (f >= 0 && f < m.nFaces) m.bPatch[f] = (int)k + 1;
  // cell -> faces: owned faces ascending, then neighbour faces ascending (main.cu:588-590)
  std::vector<int> cnt(m.nCells + 1, 0);
  for (int f = 0; f < m.nFaces; ++f) {
    if (m.owner[f] < 0) throw std::runtime_error("negative owner label at face " + std::to_string(f));
    cnt[m.owner[f] + 1]++;
  }
  for (int f = 0; f < m.nInternalFaces; ++f) {
    if (m.neigh[f] < 0) throw std::runtime_error("negative neighbour label at face " + std::to_string(f));
    cnt[m.neigh[f] + 1]++;
  }
  m.cellFaceOff.assign(m.nCells + 1, 0);
  for (int c = 0; c < m.nCells; ++c) m.cellFaceOff[c + 1] = m.cellFaceOff[c] + cnt[c + 1];
  m.cellFaces.assign(m.cellFaceOff[m.nCells], 0);
  m.cellFaceOri.assign(m.cellFaceOff[m.nCells], 0);
  std::vector<int> fill(m.cellFaceOff.begin(), m.cellFaceOff.end() - 1);
  for (int f = 0; f < m.nFaces; ++f) {
    int P = m.owner[f];
    m.cellFaces[fill[P]] = f;
    m.cellFaceOri[fill[P]++] = 1;
  }
  for (int f = 0; f < m.nInternalFaces; ++f) {
    int N = m.neigh[f];
    m.cellFaces[fill[N]] = f;
    m.cellFaceOri[fill[N]++] = -1;
  }
}

// main.cu:591-597, same operation order.
void compute_geometry(HostMesh& m, int nThreads) {
#ifdef _OPENMP
  if (nThreads > 0) omp_set_num_threads(nThreads);
#else
  (void)nThreads;
#endif
  const int nC = m.nCells, nF = m.nFaces;
  for (int f = 0; f < nF; ++f)
    for (int k = m.faceOff[f]; k < m.faceOff[f + 1]; ++k)
      if (m.facePts[k] < 0 || m.facePts[k] >= m.nPoints())
        throw std::runtime_error("face " + std::to_string(f) + " references a missing point");
  m.cc.assign(nC, {0, 0, 0});
  m.vol.assign(nC, 0.0);
  int badCell = -1;
#pragma omp parallel
  {
    std::vector<int> verts;
    std::vector<int> fv;
#pragma omp for schedule(static)
    for (int c = 0; c < nC; ++c) {
      verts.clear();
      for (int j = m.cellFaceOff[c]; j < m.cellFaceOff[c + 1]; ++j) {
        int f = m.cellFaces[j];
        for (int k = m.faceOff[f]; k < m.faceOff[f + 1]; ++k) verts.push_back(m.facePts[k]);
      }
      std::sort(verts.begin(), verts.end());
      verts.erase(std::unique(verts.begin(), verts.end()), verts.end());
      Vec3 c0{0, 0, 0};
      for (int v : verts) c0 = add3(c0, m.points[v]);
      c0 = mul3(1.0 / std::max((int)verts.size(), 1), c0);
      double V = 0.0;
      Vec3 M{0, 0, 0};
      for (int j = m.cellFaceOff[c]; j < m.cellFaceOff[c + 1]; ++j) {
        int f = m.cellFaces[j];
        fv.assign(m.facePts.begin() + m.faceOff[f], m.facePts.begin() + m.faceOff[f + 1]);
        if (m.cellFaceOri[j] < 0) std::reverse(fv.begin(), fv.end());
        const Vec3 a = m.points[fv[0]];
        for (size_t i = 1; i + 1 < fv.size(); ++i) {
          const Vec3 b = m.points[fv[i]], d = m.points[fv[i + 1]];
          double vTet = dot3(sub3(a, c0), cross3(sub3(b, c0), sub3(d, c0))) / 6.0;
          Vec3 cTet = mul3(0.25, add3(add3(c0, a), add3(b, d)));
          V += vTet;
          M = add3(M, mul3(vTet, cTet));
        }
      }
      if (V <= 0) {
#pragma omp critical
        if (badCell < 0 || c < badCell) badCell = c;
      } else {
        m.vol[c] = V;
        m.cc[c] = mul3(1.0 / V, M);
      }
    }
  }
  if (badCell >= 0) throw std::runtime_error("Non-positive cell volume at cell " + std::to_string(badCell));
  m.xf.assign(nF, {0, 0, 0});
  m.Af.assign(nF, 0.0);
  m.nf.assign(nF, {0, 0, 0});
  m.Sf.assign(nF, {0, 0, 0});
  int badFace = -1;
#pragma omp parallel for schedule(static)
  for (int f = 0; f < nF; ++f) {
    const int b0 = m.faceOff[f], nv = m.faceOff[f + 1] - b0;
    Vec3 xfc{0, 0, 0};
    for (int k = 0; k < nv; ++k) xfc = add3(xfc, m.points[m.facePts[b0 + k]]);
    xfc = mul3(1.0 / std::max(nv, 1), xfc);
    m.xf[f] = xfc;
    const Vec3 a = m.points[m.facePts[b0]];
    Vec3 areaVec{0, 0, 0};
    for (int i = 1; i + 1 < nv; ++i) {
      const Vec3 b = m.points[m.facePts[b0 + i]], d = m.points[m.facePts[b0 + i + 1]];
      areaVec = add3(areaVec, mul3(0.5, cross3(sub3(b, a), sub3(d, a))));
    }
    double areaMag = norm3(areaVec);
    if (areaMag <= 1e-30) {
#pragma omp critical
      if (badFace < 0 || f < badFace) badFace = f;
      continue;
    }
    Vec3 nloc = mul3(1.0 / areaMag, areaVec);
    const int P = m.owner[f];
    Vec3 dtest = (f < m.nInternalFaces) ? sub3(m.cc[m.neigh[f]], m.cc[P]) : sub3(m.xf[f], m.cc[P]);
    if (dot3(nloc, dtest) < 0) nloc = mul3(-1.0, nloc);
    m.Af[f] = areaMag;
    m.nf[f] = nloc;
    m.Sf[f] = mul3(areaMag, nloc);
  }
  if (badFace >= 0) throw std::runtime_error("Degenerate face area at face " + std::to_string(badFace));
  max_nonorth_deg(m);
}

void max_nonorth_deg(HostMesh& m) {
  double mx = 0.0;
#pragma omp parallel for reduction(max : mx) schedule(static)
  for (int f = 0; f < m.nInternalFaces; ++f) {
    Vec3 d = sub3(m.cc[m.neigh[f]], m.cc[m.owner[f]]);
    double cosang = std::fabs(dot3(d, m.nf[f])) / std::max(norm3(d), 1e-30);
    cosang = std::min(1.0, std::max(0.0, cosang));
    mx = std::max(mx, std::acos(cosang) * 180.0 / M_PI);
  }
  m.maxNonOrthDeg = mx;
}

HostMesh read_polymesh(const std::string& dir) {
  HostMesh m;
  auto clk = std::chrono::steady_clock::now();
  double sec[5];
  auto lap = [&](int k) {
    const auto t = std::chrono::steady_clock::now();
    sec[k] = std::chrono::duration<double>(t - clk).count();
    clk = t;
  };
  m.patches = read_boundary(dir + "/boundary");
  m.points = read_points(dir + "/points");
  lap(0);
  read_faces(dir + "/faces", m.faceOff, m.facePts);
  lap(1);
  m.owner = read_labels(dir + "/owner");
  m.neigh = read_labels(dir + "/neighbour");
  lap(2);
  finalize_topology(m);
  lap(3);
  compute_geometry(m);
  lap(4);
  if (std::getenv("ANB_SETUP_VERBOSE"))
    std::fprintf(stderr, "read_polymesh: points %.3f s, faces %.3f s, labels %.3f s, topology %.3f s, geometry %.3f s\n",
                 sec[0], sec[1], sec[2], sec[3], sec[4]);
  return m;
}

void write_polymesh(const HostMesh& m, const std::string& dir) {
  mkdir_p(dir);
  const int nF = (int)m.faceOff.size() - 1;
  std::string note = "nPoints:" + std::to_string(m.points.size()) + "  nCells:" + std::to_string(m.nCells) +
                     "  nFaces:" + std::to_string(nF) + "  nInternalFaces:" + std::to_string(m.neigh.size());
  {
    std::FILE* fp = std::fopen((dir + "/points").c_str(), "w");
    if (!fp) throw std::runtime_error("Could not open " + dir + "/points for writing");
    std::ostringstream h;
    write_header(h, "vectorField", "points", "");
    std::fputs(h.str().c_str(), fp);
    std::fprintf(fp, "%zu\n(\n", m.points.size());
    for (const auto& p : m.points) std::fprintf(fp, "(%.17g %.17g %.17g)\n", p[0], p[1], p[2]);
    std::fputs(")\n", fp);
    std::fclose(fp);
  }
  {
    std::FILE* fp = std::fopen((dir + "/faces").c_str(), "w");
    if (!fp) throw std::runtime_error("Could not open " + dir + "/faces for writing");
    std::ostringstream h;
    write_header(h, "faceList", "faces", "");
    std::fputs(h.str().c_str(), fp);
    std::fprintf(fp, "%d\n(\n", nF);
    for (int f = 0; f < nF; ++f) {
      std::fprintf(fp, "%d(", m.faceOff[f + 1] - m.faceOff[f]);
      for (int k = m.faceOff[f]; k < m.faceOff[f + 1]; ++k)
        std::fprintf(fp, k + 1 < m.faceOff[f + 1] ? "%d " : "%d", m.facePts[k]);
      std::fputs(")\n", fp);
    }
    std::fputs(")\n", fp);
    std::fclose(fp);
  }
  auto write_labels = [&](const char* obj, const std::vector<int>& v, size_t n) {
    std::FILE* fp = std::fopen((dir + "/" + obj).c_str(), "w");
    if (!fp) throw std::runtime_error(std::string("Could not open ") + dir + "/" + obj + " for writing");
    std::ostringstream h;
    write_header(h, "labelList", obj, note);
    std::fputs(h.str().c_str(), fp);
    std::fprintf(fp, "%zu\n(\n", n);
    for (size_t i = 0; i < n; ++i) std::fprintf(fp, "%d\n", v[i]);
    std::fputs(")\n", fp);
    std::fclose(fp);
  };
  write_labels("owner", m.owner, (size_t)nF);
  write_labels("neighbour", m.neigh, m.neigh.size());
  {
    std::ofstream o(dir + "/boundary");
    if (!o) throw std::runtime_error("Could not open " + dir + "/boundary for writing");
    write_header(o, "polyBoundaryMesh", "boundary", "");
    o << m.patches.size() << "\n(\n";
    for (const auto& p : m.patches) {
      o << "    " << p.name << "\n    {\n        type            " << (p.type.empty() ? "patch" : p.type)
        << ";\n        physicalType    patch;\n        nFaces          " << p.nFaces
        << ";\n        startFace       " << p.start << ";\n    }\n";
    }
    o << ")\n";
  }
}

// ---------------------------------------------------------------------------------------
// Synthetic channel meshes
// ---------------------------------------------------------------------------------------
namespace {

struct RawFace {
  int owner, neigh, patch;  // neigh = -1 for boundary; patch index for boundary faces
  int v[4];
  int nv;
};

void assemble_faces(HostMesh& m, std::vector<RawFace>& faces, int nPatches, const char* const* names) {
  std::vector<RawFace> internal, bnd;
  for (auto& f : faces) (f.neigh >= 0 ? internal : bnd).push_back(f);
  std::sort(internal.begin(), internal.end(), [](const RawFace& a, const RawFace& b) {
    return a.owner != b.owner ? a.owner < b.owner : a.neigh < b.neigh;
  });
  std::stable_sort(bnd.begin(), bnd.end(), [](const RawFace& a, const RawFace& b) {
    return a.patch != b.patch ? a.patch < b.patch : a.owner < b.owner;
  });
  m.faceOff.assign(1, 0);
  m.facePts.clear();
  m.owner.clear();
  m.neigh.clear();
  for (auto& f : internal) {
    for (int k = 0; k < f.nv; ++k) m.facePts.push_back(f.v[k]);
    m.faceOff.push_back((int)m.facePts.size());
    m.owner.push_back(f.owner);
    m.neigh.push_back(f.neigh);
  }
  m.patches.assign(nPatches, PatchInfo{});
  for (int p = 0; p < nPatches; ++p) {
    m.patches[p].name = names[p];
    m.patches[p].type = "patch";
  }
  int cursor = (int)internal.size();
  for (int p = 0; p < nPatches; ++p) m.patches[p].start = cursor;
  for (auto& f : bnd) {
    for (int k = 0; k < f.nv; ++k) m.facePts.push_back(f.v[k]);
    m.faceOff.push_back((int)m.facePts.size());
    m.owner.push_back(f.owner);
    m.patches[f.patch].nFaces++;
  }
  for (int p = 0; p < nPatches; ++p) {
    m.patches[p].start = cursor;
    cursor += m.patches[p].nFaces;
  }
}

}  // namespace

HostMesh make_channel_mesh(const ChannelSpec& s) {
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  if (nx < 1 || ny < 1 || nz < 1) throw std::runtime_error("channel mesh needs nx, ny, nz >= 1");
  const double dx = s.Lx / nx, dy = s.Ly / ny, dz = s.Lz / nz;
  auto nodeId = [&](int i, int j, int k) { return (k * (ny + 1) + j) * (nx + 1) + i; };
  // obstacle cell-index box from unjittered cell centres
  int i0 = 0, i1 = 0, j0 = 0, j1 = 0;
  if (s.obstacle) {
    i0 = nx; i1 = -1; j0 = ny; j1 = -1;
    for (int i = 0; i < nx; ++i) {
      double xc = (i + 0.5) * dx;
      if (xc >= s.ox0 && xc <= s.ox1) { i0 = std::min(i0, i); i1 = std::max(i1, i + 1); }
    }
    for (int j = 0; j < ny; ++j) {
      double yc = (j + 0.5) * dy;
      if (yc >= s.oy0 && yc <= s.oy1) { j0 = std::min(j0, j); j1 = std::max(j1, j + 1); }
    }
    if (i1 <= i0 || j1 <= j0) throw std::runtime_error("obstacle block contains no cell centre");
  }
  auto solid = [&](int i, int j, int) {
    return s.obstacle && i >= i0 && i < i1 && j >= j0 && j < j1;
  };
  // node coordinates with jitter; boundary nodes move only tangentially
  const int nN = (nx + 1) * (ny + 1) * (nz + 1);
  std::vector<Vec3> X(nN);
  std::mt19937_64 rng(s.seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        double rx = U(rng), ry = U(rng), rz = U(rng);
        bool fixX = (i == 0 || i == nx), fixY = (j == 0 || j == ny), fixZ = (k == 0 || k == nz);
        if (s.obstacle) {
          bool onXFace = (i == i0 || i == i1) && j >= j0 && j <= j1;
          bool onYFace = (j == j0 || j == j1) && i >= i0 && i <= i1;
          fixX = fixX || onXFace;
          fixY = fixY || onYFace;
        }
        Vec3 p{i * dx, j * dy, k * dz};
        if (i == nx) p[0] = s.Lx;
        if (j == ny) p[1] = s.Ly;
        if (k == nz) p[2] = s.Lz;
        if (s.jitter > 0.0) {
          if (!fixX) p[0] += s.jitter * dx * rx;
          if (!fixY) p[1] += s.jitter * dy * ry;
          if (!fixZ) p[2] += s.jitter * dz * rz;
        }
        X[nodeId(i, j, k)] = p;
      }
  // hex cell ids
  std::vector<int> hexId((size_t)nx * ny * nz, -1);
  int nHex = 0;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
        if (!solid(i, j, k)) hexId[((size_t)k * ny + j) * nx + i] = nHex++;
  auto hid = [&](int i, int j, int k) -> int {
    if (i < 0 || j < 0 || k < 0 || i >= nx || j >= ny || k >= nz) return -2;  // outside box
    return hexId[((size_t)k * ny + j) * nx + i];                             // -1 = solid
  };
  const char* names[4] = {"patch_0_0", "patch_1_0", "patch_2_0", "patch_3_0"};
  const int nPatches = s.obstacle ? 4 : 3;
  HostMesh m;
  std::vector<RawFace> faces;

  if (!s.tets) {
    faces.reserve((size_t)nHex * 3 + 2 * ((size_t)nx * ny + (size_t)ny * nz + (size_t)nx * nz));
    // quad with +axis normal at node plane; a = cell on the low side, b = cell on the high side
    auto quad = [&](int axis, int i, int j, int k, int v[4]) {
      if (axis == 0) { v[0] = nodeId(i, j, k); v[1] = nodeId(i, j + 1, k); v[2] = nodeId(i, j + 1, k + 1); v[3] = nodeId(i, j, k + 1); }
      else if (axis == 1) { v[0] = nodeId(i, j, k); v[1] = nodeId(i, j, k + 1); v[2] = nodeId(i + 1, j, k + 1); v[3] = nodeId(i + 1, j, k); }
      else { v[0] = nodeId(i, j, k); v[1] = nodeId(i + 1, j, k); v[2] = nodeId(i + 1, j + 1, k); v[3] = nodeId(i, j + 1, k); }
    };
    for (int axis = 0; axis < 3; ++axis) {
      const int ni = nx + (axis == 0), nj = ny + (axis == 1), nk = nz + (axis == 2);
      for (int k = 0; k < nk; ++k)
        for (int j = 0; j < nj; ++j)
          for (int i = 0; i < ni; ++i) {
            int lo = hid(i - (axis == 0), j - (axis == 1), k - (axis == 2));
            int hi = hid(i, j, k);
            RawFace f;
            f.nv = 4;
            quad(axis, i, j, k, f.v);
            if (lo >= 0 && hi >= 0) {
              f.owner = lo; f.neigh = hi; f.patch = -1;
              faces.push_back(f);
            } else if (lo >= 0 || hi >= 0) {
              int patch;
              bool outsideBox = (lo == -2 || hi == -2);
              if (!outsideBox) patch = 3;
              else if (axis == 0) patch = (lo == -2) ? 1 : 2;
              else patch = 0;
              f.neigh = -1; f.patch = patch;
              if (lo >= 0) {
                f.owner = lo;  // outward = +axis, keep order
              } else {
                f.owner = hi;  // outward = -axis, reverse
                std::reverse(f.v, f.v + 4);
              }
              faces.push_back(f);
            }
          }
    }
    m.nCells = nHex;
  } else {
    // Kuhn split: tet = path 000 -> e_a -> e_a+e_b -> 111 over the 6 axis permutations.
    static const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    struct TriKey { int a, b, c; int cell; int lf; };
    std::vector<std::array<int, 4>> tetV;
    tetV.reserve((size_t)nHex * 6);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if (hid(i, j, k) < 0) continue;
          for (int p = 0; p < 6; ++p) {
            int c[3] = {0, 0, 0};
            std::array<int, 4> tv;
            tv[0] = nodeId(i, j, k);
            for (int s2 = 0; s2 < 3; ++s2) {
              c[perms[p][s2]] = 1;
              tv[s2 + 1] = nodeId(i + c[0], j + c[1], k + c[2]);
            }
            tetV.push_back(tv);
          }
        }
    const int nTet = (int)tetV.size();
    std::vector<TriKey> keys((size_t)nTet * 4);
    static const int opp[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
#pragma omp parallel for schedule(static)
    for (int t = 0; t < nTet; ++t)
      for (int lf = 0; lf < 4; ++lf) {
        int a = tetV[t][opp[lf][0]], b = tetV[t][opp[lf][1]], c = tetV[t][opp[lf][2]];
        if (a > b) std::swap(a, b);
        if (b > c) std::swap(b, c);
        if (a > b) std::swap(a, b);
        keys[(size_t)t * 4 + lf] = {a, b, c, t, lf};
      }
    std::sort(keys.begin(), keys.end(), [](const TriKey& x, const TriKey& y) {
      if (x.a != y.a) return x.a < y.a;
      if (x.b != y.b) return x.b < y.b;
      if (x.c != y.c) return x.c < y.c;
      return x.cell < y.cell;
    });
    auto centroid = [&](int t) {
      Vec3 c{0, 0, 0};
      for (int q = 0; q < 4; ++q) c = add3(c, X[tetV[t][q]]);
      return mul3(0.25, c);
    };
    auto orient = [&](RawFace& f, int ownerTet) {
      Vec3 a = X[f.v[0]], b = X[f.v[1]], c = X[f.v[2]];
      Vec3 n = cross3(sub3(b, a), sub3(c, a));
      Vec3 fc = mul3(1.0 / 3.0, add3(add3(a, b), c));
      if (dot3(n, sub3(fc, centroid(ownerTet))) < 0) std::swap(f.v[1], f.v[2]);
    };
    auto nodeIJK = [&](int id, int& i, int& j, int& k) {
      i = id % (nx + 1);
      j = (id / (nx + 1)) % (ny + 1);
      k = id / ((nx + 1) * (ny + 1));
    };
    faces.reserve((size_t)nTet * 2 + 1024);
    for (size_t q = 0; q < keys.size();) {
      RawFace f;
      f.nv = 3;
      f.v[0] = keys[q].a; f.v[1] = keys[q].b; f.v[2] = keys[q].c; f.v[3] = -1;
      if (q + 1 < keys.size() && keys[q + 1].a == keys[q].a && keys[q + 1].b == keys[q].b &&
          keys[q + 1].c == keys[q].c) {
        f.owner = keys[q].cell; f.neigh = keys[q + 1].cell; f.patch = -1;
        orient(f, f.owner);
        faces.push_back(f);
        q += 2;
      } else {
        f.owner = keys[q].cell; f.neigh = -1;
        int ii[3], jj[3], kk[3];
        for (int r = 0; r < 3; ++r) nodeIJK(f.v[r], ii[r], jj[r], kk[r]);
        auto all = [&](const int* v, int val) { return v[0] == val && v[1] == val && v[2] == val; };
        if (all(ii, 0)) f.patch = 1;
        else if (all(ii, nx)) f.patch = 2;
        else if (all(jj, 0) || all(jj, ny) || all(kk, 0) || all(kk, nz)) f.patch = 0;
        else f.patch = 3;
        orient(f, f.owner);
        faces.push_back(f);
        q += 1;
      }
    }
    m.nCells = nTet;
  }
  assemble_faces(m, faces, nPatches, names);
  // drop unused points (those inside the removed obstacle)
  std::vector<int> used(nN, -1);
  for (int v : m.facePts) used[v] = 0;
  int np = 0;
  for (int v = 0; v < nN; ++v)
    if (used[v] == 0) used[v] = np++;
  m.points.resize(np);
  for (int v = 0; v < nN; ++v)
    if (used[v] >= 0) m.points[used[v]] = X[v];
  for (int& v : m.facePts) v = used[v];
  finalize_topology(m);
  return m;
}

}  // namespace anb
