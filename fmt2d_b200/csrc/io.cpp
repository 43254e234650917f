// Readers of the reference's input files (read_tomo2d.f90): the velocity
// mesh (read_smesh, :8-81), an interface (read_refl, :83-139) and the
// shot/receiver geometry with picks (read_geom, :141-248).  They follow
// Fortran list-directed input: each READ starts at a new line, takes its
// values from as many lines as it needs (blanks or commas between values,
// D or E exponents, r*v repeats, a slash ending the record) and drops the
// rest of its last line.  Two commas with only blanks between them (or a
// comma that opens the READ) give a null value, which leaves the Fortran
// variable unset; the readers report it as an unreadable item.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <vector>
#include "../../include/fmt2d_gpu.h"

namespace {

thread_local std::string g_io_err;

int io_fail(int code, const std::string& msg) {
  g_io_err = msg;
  return code;
}

// A file read record by record with list-directed value parsing.
class ListReader {
 public:
  explicit ListReader(const std::string& path)
      : own_(new std::ifstream(path)), in_(*own_) {}
  // A reader over text already in memory (one line read with `*` format).
  explicit ListReader(std::istream& in) : in_(in) {}
  bool ok() const { return (bool)in_; }
  int line() const { return line_; }

  // Start a READ: the next `n` values as text (a tag item is one more
  // value).  Returns false at end of file.  A slash ends the READ early; the
  // missing items come back empty, so the caller reports them as unreadable
  // (Fortran would leave those variables unset).
  bool read(std::vector<std::string>& items, int n) {
    items.clear();
    if (!next_line()) return false;
    comma_open_ = true;   // a comma before the first value is a null value
    while ((int)items.size() < n) {
      std::string tok;
      if (!next_token(tok)) {
        if (slash_) {
          items.resize((size_t)n);
          return true;
        }
        if (!next_line()) return false;
        continue;
      }
      // r*v repeats v r times
      const size_t star = tok.find('*');
      if (star != std::string::npos && star > 0 &&
          tok.find_first_not_of("0123456789") == star) {
        const int r = std::atoi(tok.substr(0, star).c_str());
        const std::string v = tok.substr(star + 1);
        for (int k = 0; k < r && (int)items.size() < n; ++k) items.push_back(v);
      } else {
        items.push_back(tok);
      }
    }
    return true;
  }

  // The next whole line (for the line-oriented interface reader).
  bool raw_line(std::string& s) {
    if (!std::getline(in_, s)) return false;
    ++line_;
    return true;
  }

 private:
  bool next_line() {
    slash_ = false;
    if (!std::getline(in_, buf_)) return false;
    ++line_;
    pos_ = 0;
    return true;
  }
  // The next item of the READ: a value, or an empty string for a null value.
  bool next_token(std::string& tok) {
    for (;;) {
      while (pos_ < buf_.size() && std::isspace((unsigned char)buf_[pos_])) ++pos_;
      if (pos_ >= buf_.size() || buf_[pos_] != ',') break;
      ++pos_;
      if (comma_open_) {   // two separating commas: a null value
        tok.clear();
        return true;
      }
      comma_open_ = true;
    }
    if (pos_ >= buf_.size()) return false;
    if (buf_[pos_] == '/') {
      slash_ = true;
      pos_ = buf_.size();
      return false;
    }
    const size_t b = pos_;
    while (pos_ < buf_.size() && !std::isspace((unsigned char)buf_[pos_]) && buf_[pos_] != ',' &&
           buf_[pos_] != '/')
      ++pos_;
    tok = buf_.substr(b, pos_ - b);
    comma_open_ = false;
    return true;
  }
  std::unique_ptr<std::istream> own_;
  std::istream& in_;
  bool comma_open_ = false;   // a comma was read since the last value
  std::string buf_;
  size_t pos_ = 0;
  int line_ = 0;
  bool slash_ = false;
};

bool to_double(std::string s, double& v) {
  for (char& c : s)
    if (c == 'd' || c == 'D') c = 'e';
  char* end = nullptr;
  v = std::strtod(s.c_str(), &end);
  return end && *end == '\0' && end != s.c_str();
}

bool to_int(const std::string& s, int& v) {
  char* end = nullptr;
  const long x = std::strtol(s.c_str(), &end, 10);
  if (!end || *end != '\0' || end == s.c_str()) return false;
  v = (int)x;
  return true;
}

}  // namespace

extern "C" {

int fmt2d_io_last_error(char* buf, int len) {
  if (!buf || len <= 0) return FMT2D_ERR_ARG;
  std::strncpy(buf, g_io_err.c_str(), (size_t)len - 1);
  buf[len - 1] = '\0';
  return FMT2D_OK;
}

int fmt2d_read_smesh(const char* path, int* nx, int* nz, double* vwater, double* vair,
                     double* xpos, double* topo, double* zrel, double* vel) {
  if (!path || !nx || !nz || !vwater) return FMT2D_ERR_ARG;
  ListReader r(path);
  if (!r.ok()) return io_fail(FMT2D_ERR_ARG, std::string("cannot open smesh file: ") + path);
  std::vector<std::string> it;
  int n1 = 0, n2 = 0;
  double vw = 0, va = 0;
  if (!r.read(it, 4) || !to_int(it[0], n1) || !to_int(it[1], n2) || !to_double(it[2], vw) ||
      !to_double(it[3], va))
    return io_fail(FMT2D_ERR_MODEL, "reading smesh header (nx, nz, vwater, vair)");
  if (n1 < 2 || n2 < 2) return io_fail(FMT2D_ERR_MODEL, "smesh grid too small (need nx, nz >= 2)");
  *nx = n1;
  *nz = n2;
  *vwater = vw;
  if (vair) *vair = va;
  if (!xpos && !topo && !zrel && !vel) return FMT2D_OK;   // sizes only
  std::vector<double> xs(n1), tp(n1), zr(n2), vv((size_t)n1 * n2);
  auto read_vec = [&](std::vector<double>& out) {
    if (!r.read(it, (int)out.size())) return false;
    for (size_t k = 0; k < out.size(); ++k)
      if (!to_double(it[k], out[k])) return false;
    return true;
  };
  if (!read_vec(xs)) return io_fail(FMT2D_ERR_MODEL, "reading xpos from smesh");
  if (!read_vec(tp)) return io_fail(FMT2D_ERR_MODEL, "reading topo from smesh");
  if (!read_vec(zr)) return io_fail(FMT2D_ERR_MODEL, "reading zpos_rel from smesh");
  for (int ix = 0; ix < n1; ++ix) {
    if (!r.read(it, n2))
      return io_fail(FMT2D_ERR_MODEL, "reading vel row for ix = " + std::to_string(ix + 1));
    for (int iz = 0; iz < n2; ++iz)
      if (!to_double(it[iz], vv[(size_t)iz * n1 + ix]))
        return io_fail(FMT2D_ERR_MODEL, "reading vel row for ix = " + std::to_string(ix + 1));
  }
  if (xpos) std::copy(xs.begin(), xs.end(), xpos);
  if (topo) std::copy(tp.begin(), tp.end(), topo);
  if (zrel) std::copy(zr.begin(), zr.end(), zrel);
  if (vel) std::copy(vv.begin(), vv.end(), vel);
  return FMT2D_OK;
}

int fmt2d_read_refl(const char* path, int* n, double* x, double* z) {
  if (!path || !n) return FMT2D_ERR_ARG;
  ListReader r(path);
  if (!r.ok()) return io_fail(FMT2D_ERR_ARG, std::string("cannot open refl file: ") + path);
  std::vector<double> xs, zs;
  std::string s;
  while (r.raw_line(s)) {
    if (s.find_first_not_of(" \t\r") == std::string::npos) continue;   // blank line
    // every non-blank line counts against the limit before it is parsed
    // (:105-109); a malformed line, or one with a null value, is skipped
    // (:110-116)
    if (xs.size() + 1 > 100000) return io_fail(FMT2D_ERR_MODEL, "refl file exceeds 100000 lines");
    std::istringstream ls(s);
    ListReader lr(ls);
    std::vector<std::string> it;
    double xv = 0, zv = 0;
    if (!lr.read(it, 2) || !to_double(it[0], xv) || !to_double(it[1], zv)) continue;
    xs.push_back(xv);
    zs.push_back(zv);
  }
  if (xs.empty()) return io_fail(FMT2D_ERR_MODEL, std::string("refl file has no valid data: ") + path);
  *n = (int)xs.size();
  if (x) std::copy(xs.begin(), xs.end(), x);
  if (z) std::copy(zs.begin(), zs.end(), z);
  return FMT2D_OK;
}

int fmt2d_read_geom(const char* path, int* nobs, int* nrec, double* obs_x, double* obs_z,
                    double* rec_x, double* rec_z, int* obs_id, int* phase, double* t_obs,
                    double* unc) {
  if (!path || !nobs || !nrec) return FMT2D_ERR_ARG;
  ListReader r(path);
  if (!r.ok()) return io_fail(FMT2D_ERR_ARG, std::string("cannot open geom file: ") + path);
  std::vector<std::string> it;
  int no = 0;
  if (!r.read(it, 1) || !to_int(it[0], no)) return io_fail(FMT2D_ERR_MODEL, "reading nobs from geom file");
  if (no < 1) return io_fail(FMT2D_ERR_MODEL, "invalid nobs from geom file: " + std::to_string(no));
  std::vector<double> ox(no), oz(no), rx, rz, to, un;
  std::vector<int> id, ph;
  for (int io = 0; io < no; ++io) {
    int nr = 0;
    if (!r.read(it, 4) || !to_double(it[1], ox[io]) || !to_double(it[2], oz[io]) ||
        !to_int(it[3], nr))
      return io_fail(FMT2D_ERR_MODEL, "reading OBS header for iobs = " + std::to_string(io + 1));
    for (int k = 0; k < nr; ++k) {
      double a, b, t, u;
      int p;
      if (!r.read(it, 6) || !to_double(it[1], a) || !to_double(it[2], b) || !to_int(it[3], p) ||
          !to_double(it[4], t) || !to_double(it[5], u))
        return io_fail(FMT2D_ERR_MODEL, "reading rec for iobs = " + std::to_string(io + 1) +
                                            " irec = " + std::to_string(k + 1));
      rx.push_back(a);
      rz.push_back(b);
      ph.push_back(p);
      to.push_back(t);
      un.push_back(u);
      id.push_back(io + 1);
    }
  }
  *nobs = no;
  *nrec = (int)rx.size();
  if (obs_x) std::copy(ox.begin(), ox.end(), obs_x);
  if (obs_z) std::copy(oz.begin(), oz.end(), obs_z);
  if (rec_x) std::copy(rx.begin(), rx.end(), rec_x);
  if (rec_z) std::copy(rz.begin(), rz.end(), rec_z);
  if (obs_id) std::copy(id.begin(), id.end(), obs_id);
  if (phase) std::copy(ph.begin(), ph.end(), phase);
  if (t_obs) std::copy(to.begin(), to.end(), t_obs);
  if (unc) std::copy(un.begin(), un.end(), unc);
  return FMT2D_OK;
}

}  // extern "C"
