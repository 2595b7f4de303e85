// Host post-processing of the transient results (see postprocess.h).  Both modules
// are text transforms (megabytes per transmitter); they stay on the host and
// reproduce the reference's files byte for byte: the same reading rules, the same
// arithmetic order, and numbers printed as the reference's scientific /
// precision-16 streams print them ("%.16e").  Numbers are read with from_chars and
// printed with to_chars (both correctly rounded, so equal to the C library's
// strtod / printf that the reference's streams use), and transmitters are
// processed on parallel host threads: the text work is what costs.
#include "postprocess.h"

#include "parallel.h"

#include <array>
#include <cctype>
#include <charconv>
#include <climits>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iterator>
#include <vector>

namespace tdem {
namespace {

std::string join(const std::string& dir, const std::string& name) { return dir + "/" + name; }

std::string read_text(const std::string& fn, std::string& text) {
  std::ifstream in(fn, std::ios::binary);
  if (!in) return "cannot open " + fn;
  text.assign(std::istreambuf_iterator<char>(in), std::istreambuf_iterator<char>());
  return "";
}

std::string write_text(const std::string& fn, const std::string& text) {
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) return "cannot write " + fn;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return (std::fclose(f) == 0 && ok) ? "" : "cannot write " + fn;
}

// appends v as "%.16e" prints it
void put_e16(std::string& out, double v) {
  char b[40];
  const auto r = std::to_chars(b, b + sizeof b, v, std::chars_format::scientific, 16);
  out.append(b, r.ptr);
}

void put_int(std::string& out, int v) {
  char b[16];
  const auto r = std::to_chars(b, b + sizeof b, v);
  out.append(b, r.ptr);
}

// Formatted extraction over a text with the reference's stream rules for
// well-formed numbers: leading white space is skipped; an integer is an optional
// sign and digits; a floating-point number is the longest run of sign, digits,
// point and exponent characters; a read that finds no number fails and every later
// read fails too; reaching the end of the text sets eof (as it does for a number
// that ends the text), and a read after eof fails.
class Scanner {
 public:
  Scanner(const char* b, const char* e) : p_(b), e_(e) {}
  bool fail() const { return fail_; }
  bool good() const { return !fail_ && !eof_; }

  Scanner& operator>>(int& v) {
    if (!skip_ws()) return *this;
    const char* q = p_;
    if (*q == '+' || *q == '-') ++q;
    const char* d = q;
    while (q < e_ && (unsigned)(*q - '0') < 10) ++q;
    if (q == d) return failed();
    long long x = 0;
    const char* s = p_ + (*p_ == '+');
    if (std::from_chars(s, q, x).ec != std::errc() || x > INT_MAX || x < INT_MIN) return failed();
    v = (int)x;
    p_ = q;
    if (p_ == e_) eof_ = true;
    return *this;
  }

  Scanner& operator>>(double& v) {
    if (!skip_ws()) return *this;
    const char* q = p_;
    if (*q == '+' || *q == '-') ++q;
    bool digits = false, dot = false;
    while (q < e_) {
      if ((unsigned)(*q - '0') < 10)
        digits = true;
      else if (*q == '.' && !dot)
        dot = true;
      else
        break;
      ++q;
    }
    if (!digits) return failed();
    if (q < e_ && (*q == 'e' || *q == 'E')) {
      const char* x = q + 1;
      if (x < e_ && (*x == '+' || *x == '-')) ++x;
      const char* xd = x;
      while (x < e_ && (unsigned)(*x - '0') < 10) ++x;
      if (x == xd) return failed();  // an exponent without digits
      q = x;
    }
    const char* s = p_ + (*p_ == '+');
    const auto r = std::from_chars(s, q, v);
    if (r.ec != std::errc() || r.ptr != q) return failed();
    p_ = q;
    if (p_ == e_) eof_ = true;
    return *this;
  }

  // rest of the line, at most n characters (istream::ignore(n, '\n'))
  void ignore_line(size_t n) {
    if (fail_ || eof_) {
      fail_ = true;
      return;
    }
    size_t k = 0;
    while (p_ < e_ && k < n) {
      ++k;
      if (*p_++ == '\n') return;
    }
    if (p_ == e_ && k < n) eof_ = true;
  }

  // a line of at most n - 1 characters, discarded (istream::getline(buf, n, '\n'))
  void skip_getline(size_t n) {
    if (fail_ || eof_) {
      fail_ = true;
      return;
    }
    const char* q = p_;
    while (q < e_ && *q != '\n' && (size_t)(q - p_) < n - 1) ++q;
    if (q < e_ && *q == '\n') {
      p_ = q + 1;
      return;
    }
    if (q == e_) {
      eof_ = true;
      if (q == p_) fail_ = true;
      p_ = q;
      return;
    }
    p_ = q;
    fail_ = true;  // line too long
  }

 private:
  const char* p_;
  const char* e_;
  bool fail_ = false, eof_ = false;

  bool skip_ws() {
    if (fail_ || eof_) {
      fail_ = true;
      return false;
    }
    while (p_ < e_ && std::isspace((unsigned char)*p_)) ++p_;
    if (p_ == e_) {
      eof_ = fail_ = true;
      return false;
    }
    return true;
  }
  Scanner& failed() {
    fail_ = true;
    return *this;
  }
};

// ---- SumNonstat3DOnly --------------------------------------------------------------

// One receiver of a result file: its header and nt rows of (t, three values).
struct Station {
  int ix = 0, iy = 0;
  double x = 0, y = 0, z = 0;
  std::vector<double> t, v[3];
};

// nrec receivers of nt rows each, read as whitespace-separated tokens: two ints,
// three coordinates, six header ints, the rest of that line, the legend line, then
// nt rows (SumNonstat3DOnly/picket.cpp:116-152).  A short or unreadable file is an
// error, as is ending on the last number without a newline (the reference's final
// stream-state check).
std::string read_stations(const std::string& fn, int nrec, int nt, std::vector<Station>& out) {
  std::string text;
  std::string e = read_text(fn, text);
  if (!e.empty()) return e;
  Scanner in(text.data(), text.data() + text.size());
  out.assign(nrec, Station());
  for (Station& s : out) {
    s.t.resize(nt);
    for (auto& c : s.v) c.resize(nt);
    int skip = 0;
    in >> s.ix >> s.iy >> s.x >> s.y >> s.z >> skip >> skip >> skip >> skip >> skip >> skip;
    in.ignore_line(1000);
    in.skip_getline(255);  // legend
    for (int k = 0; k < nt; ++k) in >> s.t[k] >> s.v[0][k] >> s.v[1][k] >> s.v[2][k];
  }
  if (!in.good()) return "error while reading " + fn;
  return "";
}

// One component of every receiver: t, 0 (normal part), anomalous, total (= anomalous)
// (SumNonstat3DOnly/picket.cpp:208-230 with Picket::CopyValuesOnlyAnomal).
std::string write_component(const std::string& fn, const std::vector<Station>& st, const std::vector<double>& t_ms,
                            int comp, const char* legend) {
  std::string out;
  out.reserve(st.size() * (200 + t_ms.size() * 96));
  for (const Station& s : st) {
    put_int(out, s.ix);
    out += ' ';
    put_int(out, s.iy);
    out += '\n';
    put_e16(out, s.x);
    out += ' ';
    put_e16(out, s.y);
    out += ' ';
    put_e16(out, s.z);
    out += "\n1\n1 1 1 1\n1\n";
    out += legend;
    out += '\n';
    for (size_t k = 0; k < t_ms.size(); ++k) {
      put_e16(out, t_ms[k]);
      out += ' ';
      put_e16(out, 0.0);
      out += ' ';
      put_e16(out, s.v[comp][k]);
      out += ' ';
      put_e16(out, s.v[comp][k]);
      out += '\n';
    }
  }
  return write_text(fn, out);
}

// n counts; as in the reference, counts missing from a short file read as 0
std::string read_ints(const std::string& fn, int n, std::vector<int>& out) {
  std::ifstream in(fn);
  if (!in) return "cannot open " + fn;
  out.assign(n, 0);
  for (int& v : out) in >> v;
  return "";
}

}  // namespace

std::string split_components(const std::string& dir) {
  // transmitters: sum of the place ranges of every profile (utils_direct_solver.cpp:26-48)
  int npls = 0;
  {
    std::ifstream in(join(dir, "group"));
    if (!in) return "cannot open group";
    int nprof = 0;
    in >> nprof;
    for (int i = 0; i < nprof; ++i) {
      int k = 0, p1 = 0, p2 = 0;
      in >> k >> p1 >> p2;
      npls += p2 - p1 + 1;
    }
  }
  double ftime = 0, ltime = 0;
  {
    std::ifstream in(join(dir, "timeintervalforprint"));
    if (!in) return "cannot open timeintervalforprint";
    in >> ftime >> ltime;
  }
  // time grid (utils_direct_solver.cpp:76-97): the printed layers are those in [ftime, ltime]
  std::vector<double> t_ms;
  {
    std::ifstream in(join(dir, "infite.0"));
    if (!in) return "cannot open infite.0";
    in.ignore(1000, '=');
    int nt = 0;
    in >> nt;
    if (nt < 0) return "infite.0: bad time count";
    for (int k = 0; k < 4; ++k) in.ignore(1000, '\n');
    for (int i = 0; i < nt; ++i) {
      if (!in.good()) return "infite.0: truncated";
      double t = 0;
      in >> t;
      in.ignore(1000, ';');
      if (t >= ftime && t <= ltime) t_ms.push_back(t * 1000.0);
    }
  }
  const int ntim = (int)t_ms.size();
  static const char* kB[3] = {"Bxall", "Byall", "Bzall"};
  static const char* kF[3] = {"Edsxall", "Edsyall", "Edsall"};
  static const char* kE[3] = {"Exall", "Eyall", "Ezall"};
  // column legends of the reference's files (SumNonstat3DOnly/main.cpp:196-206)
  static const char* kLegB[3] = {"t (ms)        Bx (mTl)     Bx (mTl)     Bx (mTl)",
                                 "t (ms)        By (mTl)     By (mTl)     By (mTl)",
                                 "t (ms)        Bz (mTl)     Bz (mTl)     Bz (mTl)"};
  static const char* kLegF[3] = {"t (ms)      Emfx (mV)   Emfx (mV)   Emfx (mV)",
                                 "t (ms)      Emfy (mV)   Emfy (mV)   Emfy (mV)",
                                 "t (ms)      Emfz (mV)   Emfz (mV)   Emfz (mV)"};
  static const char* kLegE[3] = {"t (ms)        Ex (V/m)     Ex (V/m)     Ex (V/m)",
                                 "t (ms)        Ey (V/m)     Ey (V/m)     Ey (V/m)",
                                 "t (ms)        Ez (V/m)     Ez (V/m)     Ez (V/m)"};
  auto split = [&](const char* stem, int p, int nrec, const char* const* names, const char* const* legends) {
    std::vector<Station> st;
    std::string err = read_stations(join(dir, std::string(stem) + "." + std::to_string(p + 1)), nrec, ntim, st);
    for (int c = 0; c < 3 && err.empty(); ++c)
      err = write_component(join(dir, std::string(names[c]) + "." + std::to_string(p + 1)), st, t_ms, c, legends[c]);
    return err;
  };
  // receiver counts of the B / emf files, then of the E files (SumNonstat3DOnly/main.cpp:258-381)
  std::string e;
  std::vector<int> nrec_b, nrec_e;
  for (const char* f : {"xyzVectorB", "xyzVectorE"}) {
    std::ifstream in(join(dir, f));
    if (!in) return std::string("cannot open ") + f;
  }
  if (!(e = read_ints(join(dir, "recvsb"), npls, nrec_b)).empty()) return e;
  if (!(e = read_ints(join(dir, "recvse"), npls, nrec_e)).empty()) return e;
  // transmitters on parallel threads (each writes its own files); the error
  // reported is the one the reference's order (B and emf of every transmitter,
  // then E) meets first
  std::vector<std::string> err_bf(npls), err_e(npls);
  parallel_ranges(npls, [&](int64_t p0, int64_t p1) {
    for (int p = (int)p0; p < (int)p1; ++p) {
      err_bf[p] = split("ball_anom", p, nrec_b[p], kB, kLegB);
      if (err_bf[p].empty()) err_bf[p] = split("edsall_anom", p, nrec_b[p], kF, kLegF);
      err_e[p] = split("eall_anom", p, nrec_e[p], kE, kLegE);
    }
  }, 1);
  for (const std::string& x : err_bf)
    if (!x.empty()) return x;
  for (const std::string& x : err_e)
    if (!x.empty()) return x;
  return "";
}

// ---- SummatorEDMN --------------------------------------------------------------------

namespace {

// The text of a file read line by line with the reference's istream::getline(buf,
// 1000, '\n') rules: a line longer than 999 characters puts the stream in a failed
// state (its first 999 characters are returned, later reads return empty lines);
// reading the end of the text sets eof (also for a last line without its newline,
// which is then still returned); after eof or a close every read returns "".
class LineReader {
 public:
  explicit LineReader(std::string text) : text_(std::move(text)) {}
  void getline(std::string& out) {
    out.clear();
    if (failed_) return;
    if (pos_ >= text_.size()) {
      eof_ = failed_ = true;
      return;
    }
    const size_t q = text_.find('\n', pos_);
    const size_t end = q == std::string::npos ? text_.size() : q;
    if (end - pos_ > 999) {
      out = text_.substr(pos_, 999);
      pos_ += 999;
      failed_ = true;
      return;
    }
    out.assign(text_, pos_, end - pos_);
    pos_ = end + 1;
    if (q == std::string::npos) eof_ = true;
  }
  bool eof() const { return eof_; }
  void close() { pos_ = text_.size(); }

 private:
  std::string text_;
  size_t pos_ = 0;
  bool eof_ = false, failed_ = false;
};

struct Curve {
  std::vector<double> t;
  std::vector<std::array<double, 3>> v;  // normal, anomalous, total
};

// One curve of an E file (SummatorEDMN/Picket.h:278-326).  `line` holds the curve's
// first line on entry (read ahead by the caller or the previous curve) and the line
// after the curve on exit.  A curve whose header does not parse is left empty and
// closes the file, so every later curve of that file is empty too.
void read_curve(LineReader& in, std::string& line, Curve& c) {
  auto scan = [&]() { return Scanner(line.data(), line.data() + line.size()); };
  {
    Scanner is = scan();
    int ix = 0, iy = 0;
    is >> ix >> iy;
    if (is.fail()) {
      in.close();
      return;
    }
  }
  in.getline(line);
  {
    Scanner is = scan();
    double x = 0, y = 0, z = 0;
    is >> x >> y >> z;
    if (is.fail()) {
      in.close();
      return;
    }
  }
  for (int k = 0; k < 4; ++k) in.getline(line);  // "1", "1 1 1 1", "1", legend
  while (!in.eof()) {
    in.getline(line);
    if (in.eof()) break;
    Scanner is = scan();
    double t = 0;
    std::array<double, 3> v{};
    is >> t >> v[0] >> v[1] >> v[2];
    if (is.fail()) break;
    c.t.push_back(t);
    c.v.push_back(v);
  }
}

// Line voltages with the midpoint of A and B as the station (SummatorEDMN/Picket.h:327-334).
std::string write_lines(const std::string& fn, const std::vector<std::array<double, 3>>& mid,
                        const std::vector<Curve>& curves, const char* legend) {
  std::string out;
  for (size_t i = 0; i < curves.size(); ++i) {
    put_int(out, (int)mid[i][0]);
    out += ' ';
    put_int(out, (int)mid[i][1]);
    out += '\n';
    put_e16(out, mid[i][0]);
    out += ' ';
    put_e16(out, mid[i][1]);
    out += ' ';
    put_e16(out, mid[i][2]);
    out += "\n1\n1 1 1 1\n1\n";
    out += legend;
    out += '\n';
    const Curve& c = curves[i];
    for (size_t l = 0; l < c.t.size(); ++l) {
      put_e16(out, c.t[l]);
      for (int q = 0; q < 3; ++q) {
        out += " \t";
        put_e16(out, c.v[l][q]);
      }
      out += '\n';
    }
  }
  return write_text(fn, out);
}

}  // namespace

std::string line_voltages(const std::string& dir, bool with_ddv, int profile, int place) {
  {
    std::ifstream in(join(dir, "xyzmn"));
    if (!in) return "cannot open xyzmn";
    int nlin = 0;
    in >> nlin;
    if (!nlin) return "";  // SummatorEDMN/main.cpp:282-291
  }
  const std::string tag = std::to_string(profile) + "_" + std::to_string(place);
  const std::string tag_mn = std::to_string(place + 1) + "_" + std::to_string(profile);
  std::string e, text[3];
  static const char* kE[3] = {"exall", "eyall", "ezall"};
  for (int c = 0; c < 3; ++c)
    if (!(e = read_text(join(dir, kE[c] + tag), text[c])).empty()) return e;
  std::ifstream mn(join(dir, "xyzmn" + tag_mn));
  if (!mn) return "cannot open " + join(dir, "xyzmn" + tag_mn);
  std::ifstream pts(join(dir, "xyzVectorElin" + tag_mn));
  if (!pts) return "cannot open " + join(dir, "xyzVectorElin" + tag_mn);
  int nlines = 0, npoints = 0;
  mn >> nlines;
  pts >> npoints;
  if (!mn || !pts || nlines <= 0 || npoints < 0) return "xyzmn" + tag_mn + " / xyzVectorElin" + tag_mn + ": bad counts";
  const int per_line = npoints / nlines;  // SummatorEDMN/main.cpp:104-106

  // E curves of every point of every line, in line order (SummatorEDMN/main.cpp:108-130);
  // the three files are read on their own threads
  std::vector<Curve> E[3];
  parallel_chunks(3, 3, [&](int c, int64_t, int64_t) {
    E[c].assign((size_t)nlines * per_line, Curve());
    LineReader in(std::move(text[c]));
    std::string line;
    in.getline(line);
    for (Curve& cv : E[c]) read_curve(in, line, cv);
  });

  // dV = sum of E . dl over the line's points; dl of the first point is twice the
  // distance from A (the points are the midpoints of equal segments), else the
  // distance from the previous point.  ddV subtracts the second half of the line
  // from the first (SummatorEDMN/main.cpp:134-200).
  std::vector<std::array<double, 3>> mid(nlines);
  std::vector<Curve> dv(nlines), ddv(with_ddv ? nlines : 0);
  int m = 0;
  for (int i = 0; i < nlines; ++i) {
    double a[3], b[3];
    mn >> a[0] >> a[1] >> a[2] >> b[0] >> b[1] >> b[2];
    if (!mn) return "xyzmn" + tag_mn + ": truncated";
    for (int k = 0; k < 3; ++k) mid[i][k] = 0.5 * (a[k] + b[k]);
    double prev[3] = {0, 0, 0};
    for (int j = 0; j < per_line; ++j, ++m) {
      double p[3], dl[3];
      pts >> p[0] >> p[1] >> p[2];
      if (!pts) return "xyzVectorElin" + tag_mn + ": truncated";
      for (int k = 0; k < 3; ++k) dl[k] = j ? p[k] - prev[k] : (p[k] - a[k]) * 2.0;
      for (int k = 0; k < 3; ++k) prev[k] = p[k];
      const Curve &ex = E[0][m], &ey = E[1][m], &ez = E[2][m];
      const size_t nt = ex.t.size();
      if (ey.v.size() < nt || ez.v.size() < nt)
        return "line " + std::to_string(i + 1) + " point " + std::to_string(j + 1) +
               ": the y or z curve has fewer time rows than the x curve";
      if (j && dv[i].v.size() < nt)
        return "line " + std::to_string(i + 1) + " point " + std::to_string(j + 1) +
               ": more time rows than the line's first point";
      for (size_t l = 0; l < nt; ++l) {
        std::array<double, 3> s;
        for (int q = 0; q < 3; ++q) s[q] = ex.v[l][q] * dl[0] + ey.v[l][q] * dl[1] + ez.v[l][q] * dl[2];
        if (j == 0) {
          dv[i].t.push_back(ex.t[l]);
          dv[i].v.push_back(s);
          if (with_ddv) {
            ddv[i].t.push_back(ex.t[l]);
            ddv[i].v.push_back(s);
          }
        } else {
          for (int q = 0; q < 3; ++q) dv[i].v[l][q] += s[q];
          if (j >= per_line / 2)
            for (int q = 0; q < 3; ++q) s[q] *= -1.;
          if (with_ddv)
            for (int q = 0; q < 3; ++q) ddv[i].v[l][q] += s[q];
        }
      }
    }
  }
  // column legends of the reference's files (SummatorEDMN/main.cpp:146,151)
  static const char* kLegDV =
      "         t, ms                         dVp, mV                         dVs, mV                         dV, mV";
  static const char* kLegDDV =
      "         t, ms                         ddVp, mV                         ddVs, mV                         ddV, mV";
  if (!(e = write_lines(join(dir, "edmnall" + tag), mid, dv, kLegDV)).empty()) return e;
  if (with_ddv && !(e = write_lines(join(dir, "edmoonall" + tag), mid, ddv, kLegDDV)).empty()) return e;
  return "";
}

}  // namespace tdem
