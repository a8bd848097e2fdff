// Patch-grid files and .dnd restart files (host code).
//
// Grid file (PatchGrid::readGrid, patchgrid.cpp:479-557; CartesianPatch::
// readFromFile, cartesianpatch.cpp:98-133; Patch::readFromFile, patch.cpp:
// 63-85; CodeString::buildFrom, codestring.cpp:43-100).  A sequence of
// blocks
//     <type> <comment text> { <numbers and solver codes> }
// ended by type 0 (or the end of the file).  Type 1001 is a Cartesian patch
// whose block holds: reference point xo yo zo, base vectors i (3) and j (3),
// IO scale, cell counts Ni Nj Nk, seek-layer counts of the six sides (i-min,
// i-max, j-min, j-max, k-min, k-max), lengths Lx Ly Lz, then solver codes up
// to the closing brace.  Reference point and lengths are multiplied by the
// block's IO scale times the caller's scale.  This reader takes
// axis-aligned patches only (base vectors (1,0,0) and (0,1,0)), like the
// rest of this library.  The writer emits the layout of the reference's
// grid generator (Python/drnum.py:199-244).
//
// .dnd file (PatchGrid::writeData / readData, patchgrid.cpp:559-611;
// Patch::writeData / readData, patch.cpp:776-790): a Qt QDataStream in its
// default big-endian byte order: int32 precision (8 or 4), the time as a
// float of that precision, then each patch's field values [var][i][j][k] in
// that precision, patches in grid order.  The file name is
// <base>_<count, six digits>.dnd.
#include "dn_gridio.h"

#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

struct dn_gridfile {
  std::vector<dn_patch_desc> patches;
  std::vector<std::string> codes;
  std::vector<std::string> comments;
};

namespace {

// CodeString::buildFrom: ',' ';' and newlines are blanks, runs of blanks
// collapse to one, no leading/trailing blank, leading zeroes of a code word
// are dropped (a zero code stays "0")
std::string normalise_codes(const std::string& in)
{
  std::string s;
  int blanks = 0;
  for (char c : in) {
    if (c == '\n' || c == ',' || c == ';' || std::isspace((unsigned char)c)) c = ' ';
    blanks = c == ' ' ? blanks + 1 : 0;
    if (blanks < 2) s.push_back(c);
  }
  if (!s.empty() && s.front() == ' ') s.erase(s.begin());
  if (!s.empty() && s.back() == ' ') s.pop_back();
  bool start = true;
  size_t i = 0;
  while (i + 1 < s.size()) {
    const char c0 = s[i], c1 = s[i + 1];
    if (c0 == '0' && c1 != ' ' && start) {
      s.erase(i, 1);
    } else if (c0 == ' ') {
      start = true;
      ++i;
    } else {
      start = false;
      ++i;
    }
  }
  return s;
}

void put_be32(std::string& out, uint32_t x)
{
  for (int b = 3; b >= 0; --b) out.push_back(char((x >> (8 * b)) & 0xff));
}

void put_be64(std::string& out, uint64_t x)
{
  for (int b = 7; b >= 0; --b) out.push_back(char((x >> (8 * b)) & 0xff));
}

uint64_t get_be(const unsigned char* p, int n)
{
  uint64_t x = 0;
  for (int b = 0; b < n; ++b) x = (x << 8) | p[b];
  return x;
}

} // namespace

namespace dn {

std::string dnd_file_name(const char* base, int count)
{
  char num[32];
  std::snprintf(num, sizeof num, "%06d", count);
  return std::string(base) + "_" + num + ".dnd";
}

void dnd_header(std::string& out, int prec, double time)
{
  put_be32(out, (uint32_t)prec);
  if (prec == 4) {
    const float t = (float)time;
    uint32_t u;
    std::memcpy(&u, &t, 4);
    put_be32(out, u);
  } else {
    uint64_t u;
    std::memcpy(&u, &time, 8);
    put_be64(out, u);
  }
}

void dnd_values(std::string& out, int prec, const double* v, size_t n)
{
  out.reserve(out.size() + n * prec);
  for (size_t i = 0; i < n; ++i) {
    if (prec == 4) {
      const float f = (float)v[i];
      uint32_t u;
      std::memcpy(&u, &f, 4);
      put_be32(out, u);
    } else {
      uint64_t u;
      std::memcpy(&u, &v[i], 8);
      put_be64(out, u);
    }
  }
}

bool dnd_read_file(const std::string& name, std::string& bytes)
{
  std::ifstream f(name, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  bytes = ss.str();
  return true;
}

bool dnd_parse_header(const std::string& bytes, int* prec, double* time, size_t* offset)
{
  if (bytes.size() < 4) return false;
  const unsigned char* p = reinterpret_cast<const unsigned char*>(bytes.data());
  const int pr = (int)(int32_t)get_be(p, 4);
  // readData takes any value other than 4 as double precision (patchgrid.cpp:589-594)
  const int q = pr == 4 ? 4 : 8;
  if (bytes.size() < (size_t)(4 + q)) return false;
  if (q == 4) {
    const uint32_t u = (uint32_t)get_be(p + 4, 4);
    float t;
    std::memcpy(&t, &u, 4);
    *time = t;
  } else {
    const uint64_t u = get_be(p + 4, 8);
    std::memcpy(time, &u, 8);
  }
  *prec = q;
  *offset = 4 + q;
  return true;
}

void dnd_get_values(const std::string& bytes, size_t offset, int prec, double* v, size_t n)
{
  const unsigned char* p = reinterpret_cast<const unsigned char*>(bytes.data()) + offset;
  for (size_t i = 0; i < n; ++i) {
    if (prec == 4) {
      const uint32_t u = (uint32_t)get_be(p + 4 * i, 4);
      float f;
      std::memcpy(&f, &u, 4);
      v[i] = f;
    } else {
      const uint64_t u = get_be(p + 8 * i, 8);
      std::memcpy(&v[i], &u, 8);
    }
  }
}

bool dnd_write_file(const std::string& name, const std::string& bytes)
{
  std::ofstream f(name, std::ios::binary | std::ios::trunc);
  if (!f) return false;
  f.write(bytes.data(), (std::streamsize)bytes.size());
  return (bool)f;
}

} // namespace dn

extern "C" {

int dn_grid_read(const char* path, double scale, dn_gridfile** out)
{
  if (!path || !out) return DN_ERR_ARG;
  *out = nullptr;
  std::ifstream f(path);
  if (!f) return DN_ERR_ARG;
  dn_gridfile* g = new dn_gridfile();
  while (true) {
    long long type = 0;
    if (!(f >> type) || type == 0) break;                   // end marker or end of file
    std::string comment;
    char c;
    bool open = false;
    while (f.get(c)) {
      if (c == '{') { open = true; break; }
      comment.push_back(c);
    }
    std::string body;
    bool closed = false;
    while (open && f.get(c)) {
      if (c == '}') { closed = true; break; }
      body.push_back(std::isspace((unsigned char)c) ? ' ' : c);
    }
    if (!open || !closed || type != 1001) {                  // unknown type or a block without braces
      delete g;
      return DN_ERR_ARG;
    }
    std::istringstream iss(body);
    double xo[3], bi[3], bj[3], io_scale, L[3];
    long long n[3], seek[6];
    bool ok = true;
    for (double& x : xo) ok = ok && (bool)(iss >> x);
    for (double& x : bi) ok = ok && (bool)(iss >> x);
    for (double& x : bj) ok = ok && (bool)(iss >> x);
    ok = ok && (bool)(iss >> io_scale);
    for (long long& x : n) ok = ok && (bool)(iss >> x);
    for (long long& x : seek) ok = ok && (bool)(iss >> x);
    for (double& x : L) ok = ok && (bool)(iss >> x);
    const bool aligned = bi[0] == 1 && bi[1] == 0 && bi[2] == 0 && bj[0] == 0 && bj[1] == 1 && bj[2] == 0;
    for (long long x : n) ok = ok && x >= 1 && x <= (1LL << 30);
    for (long long x : seek) ok = ok && x >= 0 && x <= 64;
    if (!ok || !aligned) {
      delete g;
      return DN_ERR_ARG;
    }
    std::string rest((std::istreambuf_iterator<char>(iss)), std::istreambuf_iterator<char>());
    // Patch::readFromFile: m_IOScale = file scale * caller scale, applied to
    // the reference point and the lengths
    const double s = io_scale * scale;
    dn_patch_desc d;
    std::memset(&d, 0, sizeof d);
    d.ni = (int32_t)n[0]; d.nj = (int32_t)n[1]; d.nk = (int32_t)n[2];
    for (int a = 0; a < 3; ++a) {
      d.face[a] = DN_FACE_CLOSED;
      d.origin[a] = xo[a] * s;
      d.length[a] = L[a] * s;
    }
    d.dx = d.length[0] / d.ni; d.dy = d.length[1] / d.nj; d.dz = d.length[2] / d.nk;
    for (int a = 0; a < 6; ++a) d.seek[a] = (int32_t)seek[a];
    d.add_protect = 0;
    g->patches.push_back(d);
    g->codes.push_back(normalise_codes(rest));
    g->comments.push_back(comment);
  }
  *out = g;
  return DN_OK;
}

int dn_gridfile_count(const dn_gridfile* g, int* n)
{
  if (!g || !n) return DN_ERR_ARG;
  *n = (int)g->patches.size();
  return DN_OK;
}

int dn_gridfile_patch(const dn_gridfile* g, int i, dn_patch_desc* desc, char* codes, size_t n_codes)
{
  if (!g || i < 0 || i >= (int)g->patches.size()) return DN_ERR_ARG;
  if (desc) *desc = g->patches[i];
  if (codes && n_codes) {
    std::snprintf(codes, n_codes, "%s", g->codes[i].c_str());
    if (g->codes[i].size() + 1 > n_codes) return DN_ERR_RANGE;
  }
  return DN_OK;
}

int dn_gridfile_destroy(dn_gridfile* g)
{
  delete g;
  return DN_OK;
}

int dn_grid_write(const char* path, int n, const dn_patch_desc* patches, const char* const* codes)
{
  if (!path || n < 0 || (n > 0 && !patches)) return DN_ERR_ARG;
  std::ostringstream o;
  o.precision(17);
  for (int p = 0; p < n; ++p) {
    const dn_patch_desc& d = patches[p];
    o << "1001 // index=" << p << "\n{\n";
    o << "  " << d.origin[0] << " " << d.origin[1] << " " << d.origin[2] << "\n";
    o << "  1 0 0\n  0 1 0\n  1\n";
    o << "  " << d.ni << " " << d.nj << " " << d.nk << "\n";
    o << " ";
    for (int a = 0; a < 6; ++a) o << " " << d.seek[a];
    o << "\n";
    o << "  " << d.length[0] << " " << d.length[1] << " " << d.length[2] << "\n";
    o << "  " << (codes && codes[p] ? codes[p] : "fx fy fz 0 0 0 0 0 0 0") << "\n";
    o << "}\n";
  }
  o << "0\n";
  std::ofstream f(path, std::ios::trunc);
  if (!f) return DN_ERR_ARG;
  f << o.str();
  return f ? DN_OK : DN_ERR_ARG;
}

} // extern "C"
