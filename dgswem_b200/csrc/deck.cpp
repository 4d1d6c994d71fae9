// deck.cpp -- standalone input path of libdgswem_cuda: reads an ADCIRC/DG-SWEM
// input deck (fort.14, fort.15, fort.dg, fort.13) and performs the part of
// READ_INPUT and PREP_DG that the hydro step depends on, producing the arrays
// of a dgswem_cuda_setup in the reference's Fortran layout (1-based ids,
// column-major).  This is the path a run without a Fortran host takes; with a
// Fortran host, the host passes its own PREP_DG arrays instead.
//
// Reference routines restated here:
//   read_input.F:209-3935   fort.15 / fort.14 positional reading
//   read_fort_dg.F90        fort.dg keyword and fixed formats
//   nodalattr.F:295-740     fort.13 (mannings_n_at_sea_floor)
//   prep_DG.F:1551-1990     RK_TIME (SSP tables, DTVD)
//   create_edge_data.F      edge numbering and boundary edge lists
//   count_edges.cpp         node-pair -> edge lookup
//   prep_DG.F:371-377, 978-985, 1214-1274   HB modes, CORI_EL/FRIC_EL, wet/dry init
//   prep_DG.F:180-245       EMO_DG/EFA_DG, QNAM_DG/QNPH_DG rearrangement
#include "dgswem_cuda.h"
#include "abi_util.h"

#include <algorithm>
#include <cctype>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <string_view>
#include <system_error>
#include <unordered_map>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kPi = 3.141592653589793;
constexpr double kDegToRad = kPi / 180.0;
constexpr double kEarthRadius = 6378206.4;

// A file read as Fortran list-directed records: the whole file in one
// buffer, records as (offset, length) pairs, fields as views into the buffer
// (the node and element loops of a 2M-element fort.14 allocate nothing).
class ListStream {
 public:
  bool load(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    path_ = path;
    in.seekg(0, std::ios::end);
    const std::streamoff size = in.tellg();
    in.seekg(0, std::ios::beg);
    buf_.resize(size > 0 ? (size_t)size : 0);
    if (size > 0) in.read(&buf_[0], size);
    // records: the text between line feeds (a trailing carriage return
    // dropped; a last line without a line feed is a record too).  The line
    // feeds are found in parallel, one contiguous chunk per thread, and the
    // records assembled in order.
    const size_t n = buf_.size();
    int nchunk = 1;
#ifdef _OPENMP
    nchunk = std::max(1, omp_get_max_threads());
#endif
    const size_t chunk = (n + nchunk - 1) / std::max<size_t>(nchunk, 1);
    std::vector<std::vector<size_t>> feeds(nchunk);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nchunk; ++c) {
      const size_t b = std::min(n, (size_t)c * chunk), e = std::min(n, b + chunk);
      for (size_t i = b; i < e;) {
        const void* p = std::memchr(buf_.data() + i, '\n', e - i);
        if (!p) break;
        const size_t j = (size_t)(static_cast<const char*>(p) - buf_.data());
        feeds[c].push_back(j);
        i = j + 1;
      }
    }
    size_t total = 0;
    for (const auto& f : feeds) total += f.size();
    rec_.reserve(total + 1);
    size_t start = 0;
    auto add = [&](size_t end) {
      size_t len = end - start;
      if (len > 0 && buf_[start + len - 1] == '\r') --len;
      rec_.push_back({start, len});
    };
    for (const auto& f : feeds)
      for (size_t j : f) {
        add(j);
        start = j + 1;
      }
    if (start < n) add(n);
    return true;
  }
  const std::string& path() const { return path_; }
  // random access to the records (for parsing tables in parallel)
  size_t pos() const { return next_; }
  size_t remaining() const { return rec_.size() - next_; }
  std::string_view rec(size_t i) const { return std::string_view(buf_.data() + rec_[i].first, rec_[i].second); }
  void seek(size_t i) { next_ = i; }
  // the first n fields of one record (false if it has fewer: the READ would
  // continue on the next record)
  static bool split_fields(std::string_view s, size_t n, std::string_view* out) {
    size_t got = 0, i = 0, len = s.size();
    while (i < len && got < n) {
      while (i < len && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
      if (i >= len || s[i] == '/') break;
      size_t j = i;
      while (j < len && !std::isspace((unsigned char)s[j]) && s[j] != ',' && s[j] != '/') ++j;
      out[got++] = s.substr(i, j - i);
      i = j;
      if (i < len && s[i] == '/') break;
    }
    return got == n;
  }
  std::vector<std::string> records() const {
    std::vector<std::string> out;
    out.reserve(rec_.size());
    for (const auto& r : rec_) out.emplace_back(buf_, r.first, r.second);
    return out;
  }
  std::string_view record_view() {
    if (next_ >= rec_.size()) throw dgswem::Failure(DGSWEM_ERR_IO, "premature end of " + path_);
    const auto& r = rec_[next_++];
    return std::string_view(buf_.data() + r.first, r.second);
  }
  std::string record() { return std::string(record_view()); }
  // fields of a record up to a '/' (end of the READ), blanks and commas separate
  template <typename Out>
  static void tokens(std::string_view s, Out* out) {
    size_t i = 0, n = s.size();
    while (i < n) {
      while (i < n && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
      if (i >= n || s[i] == '/') return;
      size_t j = i;
      while (j < n && !std::isspace((unsigned char)s[j]) && s[j] != ',' && s[j] != '/') ++j;
      out->emplace_back(s.substr(i, j - i));
      i = j;
      if (i < n && s[i] == '/') return;
    }
  }
  // one READ(u,*) of `n` items into views: starts a new record, spills onto
  // following ones
  void read_fields(size_t n, std::string_view* out) {
    size_t got = 0;
    while (got < n) {
      std::string_view s = record_view();
      size_t i = 0, len = s.size();
      while (i < len && got < n) {
        while (i < len && (std::isspace((unsigned char)s[i]) || s[i] == ',')) ++i;
        if (i >= len || s[i] == '/') break;
        size_t j = i;
        while (j < len && !std::isspace((unsigned char)s[j]) && s[j] != ',' && s[j] != '/') ++j;
        out[got++] = s.substr(i, j - i);
        i = j;
        if (i < len && s[i] == '/') break;
      }
    }
  }
  std::vector<std::string> read(size_t n) {
    std::vector<std::string_view> v(n);
    read_fields(n, v.data());
    return std::vector<std::string>(v.begin(), v.end());
  }
  double real() {
    std::string_view v;
    read_fields(1, &v);
    return as_real(v);
  }
  int integer() {
    std::string_view v;
    read_fields(1, &v);
    return as_int(v);
  }
  // Fortran reals, including D exponents
  static double as_real(std::string_view s) {
    double v = 0.0;
    const char* b = s.data();
    const char* e = b + s.size();
    if (!s.empty() && *b == '+') ++b;
    auto r = std::from_chars(b, e, v);
    if (r.ec == std::errc() && r.ptr == e) return v;
    std::string t(s);
    for (char& c : t)
      if (c == 'd' || c == 'D') c = 'e';
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) throw dgswem::Failure(DGSWEM_ERR_IO, "expected a real, got '" + t + "'");
    return v;
  }
  static int as_int(std::string_view s) {
    long v = 0;
    const char* b = s.data();
    const char* e = b + s.size();
    if (!s.empty() && *b == '+') ++b;
    auto r = std::from_chars(b, e, v);
    if (r.ec != std::errc() || r.ptr == b) throw dgswem::Failure(DGSWEM_ERR_IO, "expected an integer, got '" + std::string(s) + "'");
    return (int)v;
  }

 private:
  std::string path_;
  std::string buf_;
  std::vector<std::pair<size_t, size_t>> rec_;
  size_t next_ = 0;
};

std::string trimmed(const std::string& s) {
  size_t b = s.find_first_not_of(" \t");
  if (b == std::string::npos) return std::string();
  size_t e = s.find_last_not_of(" \t");
  return s.substr(b, e - b + 1);
}

// A table of `count` READs of `nf` fields starting at the stream's position,
// one record each in well-formed decks: parsed by `row(i, fields)` on all
// host threads (rows must write disjoint outputs); if a record has fewer
// fields or `row` throws, the whole table is parsed again sequentially, which
// reports the error as the one-READ-at-a-time reading would.
template <int NF, typename Row>
void parse_table(ListStream& f, int count, Row row) {
  const size_t r0 = f.pos();
  int bad = 0;
  if (f.remaining() >= (size_t)count) {
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int i = 0; i < count; ++i) {
      if (bad) continue;
      std::string_view t[NF];
      if (!ListStream::split_fields(f.rec(r0 + i), NF, t)) {
        bad = 1;
        continue;
      }
      try {
        row(i, t);
      } catch (...) {
        bad = 1;
      }
    }
    if (!bad) {
      f.seek(r0 + count);
      return;
    }
  }
  f.seek(r0);
  for (int i = 0; i < count; ++i) {
    std::string_view t[NF];
    f.read_fields(NF, t);
    row(i, t);
  }
}

// One land/flow/barrier boundary segment of fort.14 after READ_INPUT's
// processing (island closing, barrier side swap).
struct Segment {
  int ibtype = 0;
  std::vector<int> nodes;                  // NBVV(K,1:NVELL), 1-based
};

}  // namespace

struct dgswem_deck {
  dgswem_cuda_setup s{};
  // run controls
  int nt = 0, noutge = 0, nspoolge = 0, ntcysge = 0, ntcyfge = 0;
  // fort.dg
  int ph = 1, pl = 1, rk_stage = 2, rk_order = 2, modal_ic = 0, artdif = 0, sedflag = 0;
  int dghot = 0, dghotspool = 86400, hot_it = 0;  // DG hot start output switch / interval; ITHS read
  // storage the setup points into
  std::vector<double> atvd, btvd, dtvd;
  std::vector<int> nm, nedno, nedel, nedsd, neled;
  std::vector<int> niedn, nledn, needn, nfedn, nredn, nebsegn, nibsegn;
  std::vector<double> x, y, dp, sfea, hb, cori_el, fric_el, manning;
  std::vector<double> ze, qx, qy;
  std::vector<int> wdflg;
  std::vector<double> amig, ff, face, per, emo_dg, efa_dg;
  std::vector<double> famig, fff, fface, fper, qnam_dg, qnph_dg;
  std::vector<double> ebht, ebcfsp, ibht, ibcfsb, ibcfsp;
};

namespace {

struct Fort15 {
  int nolibf = 0, nolica = 0, nolicat = 0, nwp = 0, ncor = 0, ntip = 0, nws = 0;
  int im = 0, nfover = 0, nstartdry = 0;
  double cori = 0, tau = 0, slam0 = 0, rnday = 0;
  bool manning = false;
  int nbfr = 0;
  std::vector<std::vector<double>> emo, efa;  // [freq][open-boundary node]
  std::vector<std::vector<int>> open_segments;  // NBDV, 1-based
  std::vector<Segment> segments;
  // node lists of READ_INPUT's boundary bookkeeping (NBV, IBCONN, LBCODEI)
  std::vector<int> nbv, ibconn, lbcodei;
  std::vector<std::pair<int, int>> backnodes;
  int nffr = 0;
  std::vector<std::vector<double>> qnam, qnph;
};

void read_fort_dg(const std::string& dir, dgswem_deck* d) {
  ListStream f;
  if (!f.load(dir + "/fort.dg")) throw dgswem::Failure(DGSWEM_ERR_IO, "cannot open " + dir + "/fort.dg");
  std::vector<std::string> first;
  if (!f.records().empty()) ListStream::tokens(f.records()[0], &first);
  if (!first.empty() && first[0][0] == '1') {  // fixed format, read_fort_dg.F90:96-150
    f.read(1);
    f.read(2);
    f.read(2);
    auto p = f.read(3);
    d->pl = ListStream::as_int(p[0]);
    d->ph = ListStream::as_int(p[1]);
    f.read(1); f.read(1); f.read(3);
    f.read(1);  // fluxtype (the LLF flux is compiled in regardless)
    auto rk = f.read(2);
    d->rk_stage = ListStream::as_int(rk[0]);
    d->rk_order = ListStream::as_int(rk[1]);
    f.read(1);
    d->modal_ic = f.integer();
    {
      auto h = f.read(2);  // DGHOT, DGHOTSPOOL (read_fort_dg.F90:111)
      d->dghot = ListStream::as_int(h[0]);
      d->dghotspool = ListStream::as_int(h[1]);
    }
    d->s.slopeflag = f.integer();
    d->sedflag = ListStream::as_int(f.read(4)[0]);
    f.read(1); f.read(1);
    d->artdif = ListStream::as_int(f.read(5)[0]);
    return;
  }
  // keyword format (read_fort_dg.F90:186-300), defaults of FORT_DG_SETUP
  d->pl = 1; d->ph = 1; d->rk_stage = 2; d->rk_order = 2; d->modal_ic = 0; d->dghot = 0; d->dghotspool = 86400;
  d->s.slopeflag = 5; d->s.rainfall = 0; d->artdif = 0; d->sedflag = 0;
  std::unordered_map<std::string, int*> ints = {
      {"pl", &d->pl}, {"ph", &d->ph}, {"rk_stage", &d->rk_stage}, {"rk_order", &d->rk_order},
      {"modal_ic", &d->modal_ic}, {"slopeflag", &d->s.slopeflag}, {"rainfall", &d->s.rainfall},
      {"artdif", &d->artdif}, {"sedflag", &d->sedflag}, {"dghot", &d->dghot}, {"dghotspool", &d->dghotspool}};
  for (const std::string& raw : f.records()) {
    std::string line = trimmed(raw);
    if (line.empty() || line[0] == '!') continue;
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = trimmed(line.substr(0, eq));
    size_t bang = line.find('!', eq);
    std::string val = line.substr(eq + 1, bang == std::string::npos ? std::string::npos : bang - eq - 1);
    auto it = ints.find(key);
    if (it == ints.end()) continue;
    std::vector<std::string> t;
    ListStream::tokens(val, &t);
    if (!t.empty()) *it->second = ListStream::as_int(t[0]);
  }
}

void read_fort13(const std::string& dir, dgswem_deck* d) {
  ListStream f;
  if (!f.load(dir + "/fort.13")) throw dgswem::Failure(DGSWEM_ERR_IO, "NWP>0 but fort.13 is missing");
  f.record();
  if (f.integer() != d->s.np) throw dgswem::Failure(DGSWEM_ERR_IO, "fort.13 node count differs from fort.14");
  int nattr = f.integer();
  std::unordered_map<std::string, double> defaults;
  for (int k = 0; k < nattr; ++k) {
    std::string name = trimmed(f.record());
    f.record();
    int nvals = f.integer();
    defaults[name] = ListStream::as_real(f.read((size_t)nvals)[0]);
  }
  bool found = false;
  for (int k = 0; k < nattr; ++k) {
    std::string name = trimmed(f.record());
    int count = f.integer();
    bool take = name == "mannings_n_at_sea_floor";
    if (take) {
      found = true;
      d->manning.assign(d->s.np, defaults[name]);
    }
    if (!take) {
      for (int i = 0; i < count; ++i) f.record_view();
      continue;
    }
    parse_table<2>(f, count, [&](int, const std::string_view* t) {
      int node = ListStream::as_int(t[0]);
      if (node < 1 || node > d->s.np) throw dgswem::Failure(DGSWEM_ERR_IO, "fort.13 node out of range");
      d->manning[node - 1] = ListStream::as_real(t[1]);
    });
  }
  if (!found) throw dgswem::Failure(DGSWEM_ERR_IO, "fort.13 has no mannings_n_at_sea_floor data");
}

void read_fort14_15(const std::string& dir, dgswem_deck* d, Fort15* p) {
  dgswem_cuda_setup& s = d->s;
  ListStream f15, f14;
  if (!f15.load(dir + "/fort.15")) throw dgswem::Failure(DGSWEM_ERR_IO, "cannot open " + dir + "/fort.15");
  if (!f14.load(dir + "/fort.14")) throw dgswem::Failure(DGSWEM_ERR_IO, "cannot open " + dir + "/fort.14");
  f15.record();
  f15.record();
  p->nfover = f15.integer();
  f15.integer();
  f15.integer();
  if (f15.integer() != 0) throw dgswem::Failure(DGSWEM_ERR_ARG, "IHOT must be 0 (cold start)");
  s.ics = f15.integer();
  p->im = f15.integer();
  p->nolibf = f15.integer();
  s.nolifa = f15.integer();
  if (s.nolifa == 3) { s.nolifa = 2; p->nstartdry = 1; }
  p->nolica = f15.integer();
  p->nolicat = f15.integer();
  p->nwp = f15.integer();
  for (int k = 0; k < p->nwp; ++k)
    if (trimmed(f15.record()) == "mannings_n_at_sea_floor") p->manning = true;
  p->ncor = f15.integer();
  p->ntip = f15.integer();
  if (p->ntip != 0) throw dgswem::Failure(DGSWEM_ERR_ARG, "NTIP != 0 is not supported");
  int nws = f15.integer();
  if (nws != 0 && nws != 1) throw dgswem::Failure(DGSWEM_ERR_ARG, "only NWS = 0 or 1 is supported");
  s.nws = nws;
  s.nramp = f15.integer();
  s.g = f15.real();
  f15.real();  // TAU0
  s.dtdp = f15.real();
  s.statim = f15.real();
  f15.real();  // REFTIM
  p->rnday = f15.real();
  d->nt = (int)(p->rnday * (86400.0 / s.dtdp) + 0.5);
  if (s.nramp <= 1) {
    s.dramp = f15.real();
  } else if (s.nramp <= 7) {
    s.dramp = ListStream::as_real(f15.read((size_t)std::max(3, s.nramp + 1))[0]);
  } else {
    throw dgswem::Failure(DGSWEM_ERR_ARG, "NRAMP > 7");
  }
  f15.read(3);
  s.h0 = ListStream::as_real(f15.read(s.nolifa == 2 ? 4 : 1)[0]);
  f14.record();
  {
    auto t = f14.read(2);
    s.ne = ListStream::as_int(t[0]);
    s.np = ListStream::as_int(t[1]);
  }
  if (s.ne <= 0 || s.np <= 0) throw dgswem::Failure(DGSWEM_ERR_IO, "empty mesh");
  {
    auto t = f15.read(2);
    p->slam0 = ListStream::as_real(t[0]) * kDegToRad;
    s.sfea0 = ListStream::as_real(t[1]) * kDegToRad;
  }
  const int np = s.np, ne = s.ne;
  d->x.assign(np, 0.0); d->y.assign(np, 0.0); d->dp.assign(np, 0.0); d->sfea.assign(np, 0.0);
  parse_table<4>(f14, np, [&](int, const std::string_view* t) {
    int id = ListStream::as_int(t[0]);
    if (id < 1 || id > np) throw dgswem::Failure(DGSWEM_ERR_IO, "node number out of range in fort.14");
    double a = ListStream::as_real(t[1]), b = ListStream::as_real(t[2]);
    if (s.ics == 1) {
      d->x[id - 1] = a;
      d->y[id - 1] = b;
      d->sfea[id - 1] = b / kEarthRadius;
    } else {
      double lam = kDegToRad * a, phi = kDegToRad * b;
      d->x[id - 1] = kEarthRadius * (lam - p->slam0) * std::cos(s.sfea0);
      d->y[id - 1] = phi * kEarthRadius;
      d->sfea[id - 1] = phi;
    }
    d->dp[id - 1] = ListStream::as_real(t[3]);
  });
  if (s.nolifa <= 1)
    for (double& v : d->dp) v = std::max(v, s.h0);  // read_input.F:1356
  d->nm.assign(3 * (size_t)ne, 0);
  parse_table<5>(f14, ne, [&](int, const std::string_view* t) {
    int id = ListStream::as_int(t[0]);
    if (id < 1 || id > ne) throw dgswem::Failure(DGSWEM_ERR_IO, "element number out of range in fort.14");
    for (int v = 0; v < 3; ++v) {
      int n = ListStream::as_int(t[2 + v]);
      if (n < 1 || n > np) throw dgswem::Failure(DGSWEM_ERR_IO, "connectivity refers to a missing node");
      d->nm[(id - 1) + (size_t)ne * v] = n;
    }
  });
  for (int e = 0; e < ne; ++e) {  // read_input.F:1406-1419
    const double* X = d->x.data();
    const double* Y = d->y.data();
    int a = d->nm[e] - 1, b = d->nm[e + ne] - 1, c = d->nm[e + 2 * (size_t)ne] - 1;
    double area2 = (X[a] - X[c]) * (Y[b] - Y[c]) + (X[c] - X[b]) * (Y[a] - Y[c]);
    if (area2 < 0.0)
      throw dgswem::Failure(DGSWEM_ERR_IO, "element " + std::to_string(e + 1) + " is ordered clockwise");
  }
  if (p->nstartdry) throw dgswem::Failure(DGSWEM_ERR_ARG, "NOLIFA = 3 (fort.12 start-dry) is not supported");
  s.hbreak = 1.0; s.ftheta = 1.0; s.fgamma = 1.0;
  if (p->nolibf == 0) p->tau = f15.real();
  s.cf = p->tau;
  if (p->nolibf == 1) s.cf = f15.real();
  if (p->nolibf == 2) {
    auto t = f15.read(4);
    s.cf = ListStream::as_real(t[0]);
    s.hbreak = ListStream::as_real(t[1]);
    s.ftheta = ListStream::as_real(t[2]);
    s.fgamma = ListStream::as_real(t[3]);
  }
  f15.read(p->im == 10 ? 2 : 1);
  if (p->nwp > 0) {
    if (!p->manning) throw dgswem::Failure(DGSWEM_ERR_ARG, "only the Manning nodal attribute is supported");
    read_fort13(dir, d);
  }
  p->cori = f15.real();
  int ntif = f15.integer();
  for (int i = 0; i < ntif; ++i) { f15.record(); f15.read(5); }
  p->nbfr = f15.integer();
  for (int i = 0; i < p->nbfr; ++i) {
    f15.record();
    auto t = f15.read(3);
    double w = ListStream::as_real(t[0]);
    d->amig.push_back(w);
    d->ff.push_back(ListStream::as_real(t[1]));
    d->face.push_back(ListStream::as_real(t[2]) * kDegToRad);
    d->per.push_back(w == 0.0 ? 0.0 : 2.0 * kPi / w);
  }
  int nope = f14.integer();
  int neta = f14.integer();
  int count = 0;
  for (int k = 0; k < nope; ++k) {
    int nv = f14.integer();
    std::vector<int> seg;
    for (int i = 0; i < nv; ++i) seg.push_back(f14.integer());
    count += nv;
    p->open_segments.push_back(seg);
  }
  if (count != neta) {
    if (p->nfover != 1) throw dgswem::Failure(DGSWEM_ERR_IO, "NETA disagrees with the open boundary segments");
    neta = count;
  }
  if (p->nbfr == 0 && nope > 0)
    throw dgswem::Failure(DGSWEM_ERR_ARG, "aperiodic elevation boundaries (fort.19) are not supported");
  p->emo.assign(p->nbfr, std::vector<double>(neta));
  p->efa.assign(p->nbfr, std::vector<double>(neta));
  for (int f = 0; f < p->nbfr; ++f) {
    f15.record();
    for (int j = 0; j < neta; ++j) {
      auto t = f15.read(2);
      p->emo[f][j] = ListStream::as_real(t[0]);
      p->efa[f][j] = ListStream::as_real(t[1]) * kDegToRad;
    }
  }
  f15.read(1);  // ANGINN
  int nbou = f14.integer();
  f14.integer();
  bool has_flow = false;
  for (int k = 0; k < nbou; ++k) {
    auto t = f14.read(2);
    int n = ListStream::as_int(t[0]);
    int ib = ListStream::as_int(t[1]);
    const bool ext = ib == 3 || ib == 13 || ib == 23;
    const bool wall = ib == 4 || ib == 24;
    static const int kAllowed[] = {0, 10, 20, 1, 11, 21, 2, 12, 22, 3, 13, 23, 4, 24, 30};
    if (std::find(std::begin(kAllowed), std::end(kAllowed), ib) == std::end(kAllowed))
      throw dgswem::Failure(DGSWEM_ERR_ARG, "boundary type " + std::to_string(ib) + " is not supported");
    has_flow = has_flow || ib == 2 || ib == 12 || ib == 22;
    std::vector<int> node(n), partner(n, 0);
    std::vector<double> height(n), coef_sub(n), coef_sup(n);
    for (int i = 0; i < n; ++i) {
      if (ext) {
        auto r = f14.read(3);
        node[i] = ListStream::as_int(r[0]);
        height[i] = ListStream::as_real(r[1]);
        coef_sup[i] = ListStream::as_real(r[2]);
      } else if (wall) {
        auto r = f14.read(5);
        node[i] = ListStream::as_int(r[0]);
        partner[i] = ListStream::as_int(r[1]);
        height[i] = ListStream::as_real(r[2]);
        coef_sub[i] = ListStream::as_real(r[3]);
        coef_sup[i] = ListStream::as_real(r[4]);
      } else {
        node[i] = f14.integer();
      }
    }
    // internal barriers are walked twice; the second walk swaps the two sides
    // and reverses the order, which is what NBVV keeps (read_input.F:2445-2470)
    for (int pass = 0; pass < (wall ? 2 : 1); ++pass) {
      if (pass == 1) {
        std::reverse(node.begin(), node.end());
        std::reverse(partner.begin(), partner.end());
        std::swap(node, partner);
        std::reverse(height.begin(), height.end());
        std::reverse(coef_sub.begin(), coef_sub.end());
        std::reverse(coef_sup.begin(), coef_sup.end());
      }
      Segment seg;
      seg.ibtype = ib;
      seg.nodes = node;
      if ((ib == 1 || ib == 11 || ib == 21) && seg.nodes.back() != seg.nodes.front())
        seg.nodes.push_back(seg.nodes.front());  // close islands
      for (size_t i = 0; i < seg.nodes.size(); ++i) {
        p->nbv.push_back(seg.nodes[i]);
        p->lbcodei.push_back(ib);
        p->ibconn.push_back(wall ? partner[i] : 0);
      }
      if (pass == (wall ? 1 : 0)) p->segments.push_back(seg);
    }
    for (int i = 0; i + 1 < n; ++i) {  // per-segment barrier data (read_input.F:2668-2685)
      if (ext) {
        d->ebht.push_back(0.5 * (height[i] + height[i + 1]));
        d->ebcfsp.push_back(0.5 * (coef_sup[i] + coef_sup[i + 1]));
      } else if (wall) {
        d->ibht.push_back(0.5 * (height[i] + height[i + 1]));
        d->ibcfsb.push_back(0.5 * (coef_sub[i] + coef_sub[i + 1]));
        d->ibcfsp.push_back(0.5 * (coef_sup[i] + coef_sup[i + 1]));
        p->backnodes.push_back({partner[i], partner[i + 1]});
      }
    }
  }
  if (has_flow) {  // periodic flux boundaries (read_input.F:2971-3045)
    p->nffr = f15.integer();
    if (p->nffr == 0) throw dgswem::Failure(DGSWEM_ERR_ARG, "aperiodic flux boundaries (fort.20) are not supported");
    for (int i = 0; i < p->nffr; ++i) {
      f15.record();
      auto t = f15.read(3);
      double w = ListStream::as_real(t[0]);
      d->famig.push_back(w);
      d->fff.push_back(ListStream::as_real(t[1]));
      d->fface.push_back(ListStream::as_real(t[2]) * kDegToRad);
      d->fper.push_back(w == 0.0 ? 0.0 : 2.0 * kPi / w);
    }
    size_t nflow = std::count_if(p->lbcodei.begin(), p->lbcodei.end(),
                                 [](int c) { return c == 2 || c == 12 || c == 22; });
    p->qnam.assign(p->nffr, std::vector<double>(nflow));
    p->qnph.assign(p->nffr, std::vector<double>(nflow));
    for (int f = 0; f < p->nffr; ++f) {
      f15.record();
      for (size_t j = 0; j < nflow; ++j) {
        auto t = f15.read(2);
        p->qnam[f][j] = ListStream::as_real(t[0]);
        p->qnph[f][j] = ListStream::as_real(t[1]) * kDegToRad;
      }
    }
  }
  auto stations = [&]() {
    int n = f15.integer();
    for (int i = 0; i < n; ++i) f15.read(2);
  };
  f15.read(4); stations();
  f15.read(4); stations();
  if (p->im == 10) { f15.read(4); stations(); }
  if (s.nws != 0) { f15.read(4); stations(); }
  {
    auto t = f15.read(4);
    d->noutge = ListStream::as_int(t[0]);
    double ts = ListStream::as_real(t[1]), tf = ListStream::as_real(t[2]);
    d->nspoolge = ListStream::as_int(t[3]);
    d->ntcysge = (int)((ts - s.statim) * (86400.0 / s.dtdp) + 0.5);
    d->ntcyfge = std::min((int)((tf - s.statim) * (86400.0 / s.dtdp) + 0.5), d->nt);
  }
  // dgswem.F:131-170
  s.iflinbf = p->nolibf == 0 ? 1 : 0;
  s.ifhybf = p->nolibf == 2 ? 1 : 0;
  s.ifnlfa = s.nolifa == 0 ? 0 : 1;
  s.nleq = p->nolicat == 0 ? 0.0 : 1.0;  // NOLICAT is read last and wins
  s.leq = 1.0 - s.nleq;
  s.load_manning = p->manning ? 1 : 0;
}

// prep_DG.F:1551-1990 (SSP schemes of RK_TIME)
void rk_tables(dgswem_deck* d) {
  const int n = d->rk_stage, order = d->rk_order;
  if (n < 1 || n > 8) throw dgswem::Failure(DGSWEM_ERR_ARG, "rk_stage out of range");
  std::vector<double> a((size_t)n * n, 0.0), b((size_t)n * n, 0.0), c((size_t)n * n, 0.0);
  auto A = [&](int i, int j) -> double& { return a[(size_t)(i - 1) * n + (j - 1)]; };
  auto B = [&](int i, int j) -> double& { return b[(size_t)(i - 1) * n + (j - 1)]; };
  auto C = [&](int i, int j) -> double& { return c[(size_t)(i - 1) * n + (j - 1)]; };
  struct Entry { int i, j; double v; };
  auto put = [&](std::initializer_list<Entry> ea, std::initializer_list<Entry> eb) {
    for (auto& e : ea) A(e.i, e.j) = e.v;
    for (auto& e : eb) B(e.i, e.j) = e.v;
  };
  if (n == 1 && order == 1) {
    put({{1, 1, 1.0}}, {{1, 1, 1.0}});
  } else if (order == 2 && n == 3) {  // Kubatko-Yeager-Ketcheson SSP(3,2)
    put({{1, 1, 1.0}, {2, 1, 0.087353119859156}, {3, 1, 0.344956917166841},
         {2, 2, 0.912646880140844}, {3, 3, 0.655043082833159}},
        {{1, 1, 0.528005024856522}, {3, 1, 0.022826837460491}, {2, 2, 0.481882138633993},
         {3, 3, 0.345866039233415}});
  } else if (order == 2 && n == 4) {
    put({{1, 1, 1.0}, {2, 1, 0.394806441339829}, {3, 1, 0.002797307087390},
         {4, 1, 0.252860909354373}, {2, 2, 0.605193558660171}, {3, 3, 0.997202692912610},
         {4, 4, 0.747139090645627}},
        {{1, 1, 0.406584463657504}, {3, 1, 0.013637216641451}, {4, 1, 0.016453567333598},
         {2, 2, 0.246062298456822}, {3, 3, 0.405447122055692}, {4, 4, 0.303775146447707}});
  } else if (order == 2 && n == 5) {
    put({{1, 1, 1.0}, {2, 1, 0.235593265061659}, {3, 1, 0.174017972351526},
         {4, 1, 0.235264368870758}, {5, 1, 0.141720372339803}, {2, 2, 0.764406734938341},
         {4, 2, 0.000058643383967}, {5, 2, 0.095374613155521}, {3, 3, 0.825982027648475},
         {5, 3, 0.000311763705780}, {4, 4, 0.764676987745275}, {5, 5, 0.762593250798895}},
        {{1, 1, 0.324840618151514}, {3, 1, 0.108822380501601}, {4, 1, 0.054392262422093},
         {5, 1, 0.000000180291569}, {2, 2, 0.248310356296551}, {4, 2, 0.000019049753098},
         {5, 2, 0.030981548293401}, {3, 3, 0.268312512443371}, {5, 3, 0.000101273514903},
         {4, 4, 0.248398145385413}, {5, 5, 0.247721262987686}});
  } else if (order == 2) {  // generic SSP(s,2), prep_DG.F:1649-1668
    for (int i = 1; i < n; ++i) { A(i, i) = 1.0; B(i, i) = 1.0 / (n - 1); }
    A(n, 1) = 1.0 / n;
    A(n, n) = (n - 1.0) / n;
    B(n, n) = 1.0 / n;
  } else if (order == 3 && n == 3) {
    put({{1, 1, 1.0}, {2, 1, 3.0 / 4.0}, {2, 2, 1.0 / 4.0}, {3, 1, 1.0 / 3.0}, {3, 3, 2.0 / 3.0}},
        {{1, 1, 1.0}, {2, 2, 1.0 / 4.0}, {3, 3, 2.0 / 3.0}});
  } else {
    throw dgswem::Failure(DGSWEM_ERR_ARG, "unsupported rk_stage/rk_order combination");
  }
  for (int k = 0; k <= n - 1; ++k)
    for (int i = 1; i <= n; ++i) {
      double acc = 0.0;
      for (int l = k + 1; l <= i - 1; ++l) acc = acc + C(l, k + 1) * A(i, l + 1);
      C(i, k + 1) = B(i, k + 1) + acc;
    }
  d->dtvd.assign(n, 0.0);
  for (int k = 1; k <= n - 1; ++k) {
    double acc = 0.0;
    for (int l = 0; l <= k - 1; ++l) acc = acc + C(k, l + 1);
    d->dtvd[k] = acc;
  }
  d->atvd = a;
  d->btvd = b;
}

// create_edge_data.F:31-635 + count_edges.cpp, Fortran layout outputs
void build_edges(dgswem_deck* d, const Fort15& p) {
  const int ne = d->s.ne, np = d->s.np;
  auto NM = [&](int e, int v) { return d->nm[e + (size_t)ne * v]; };  // 1-based node
  std::vector<int> node_first(np + 1, 0), node_elems;
  for (int e = 0; e < ne; ++e)
    for (int v = 0; v < 3; ++v) ++node_first[NM(e, v)];
  for (int n = 1; n <= np; ++n) node_first[n] += node_first[n - 1];
  node_elems.resize(node_first[np]);
  {
    std::vector<int> cur(node_first.begin(), node_first.end() - 1);
    for (int e = 0; e < ne; ++e)
      for (int v = 0; v < 3; ++v) node_elems[cur[NM(e, v) - 1]++] = e;
  }
  d->neled.assign(3 * (size_t)ne, 0);
  d->nedno.clear();
  d->nedel.clear();
  // the first other element of node a's star (in star order) holding local
  // edge l's node pair, and its local edge: a function of the mesh alone,
  // found for every (element, edge) in parallel
  std::vector<int> match(3 * (size_t)ne, -1);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < ne; ++e)
    for (int l = 0; l < 3; ++l) {
      const int a = NM(e, (l + 1) % 3), b = NM(e, (l + 2) % 3);
      for (int q = node_first[a - 1]; q < node_first[a]; ++q) {
        const int o = node_elems[q];
        if (o == e) continue;
        int hit = -1;
        for (int m = 0; m < 3 && hit < 0; ++m) {
          const int c1 = NM(o, (m + 1) % 3), c2 = NM(o, (m + 2) % 3);
          if ((c1 == a && c2 == b) || (c1 == b && c2 == a)) hit = m;
        }
        if (hit >= 0) {
          match[l + 3 * (size_t)e] = 3 * o + hit;
          break;
        }
      }
    }
  // edge ids in the order of first visit (create_edge_data.F:85-138)
  int nedges = 0;
  for (int e = 0; e < ne; ++e) {
    for (int l = 0; l < 3; ++l) {
      if (d->neled[l + 3 * (size_t)e] != 0) continue;
      int a = NM(e, (l + 1) % 3), b = NM(e, (l + 2) % 3);
      int id = ++nedges;
      d->neled[l + 3 * (size_t)e] = id;
      d->nedno.push_back(a);
      d->nedno.push_back(b);
      d->nedel.push_back(e + 1);
      d->nedel.push_back(0);
      const int mt = match[l + 3 * (size_t)e];
      if (mt >= 0) {
        const int o = mt / 3, m = mt % 3;
        if (d->neled[m + 3 * (size_t)o] != 0)
          throw dgswem::Failure(DGSWEM_ERR_IO, "possible duplicate element " + std::to_string(o + 1));
        d->neled[m + 3 * (size_t)o] = id;
        d->nedel[2 * (size_t)(id - 1) + 1] = o + 1;
      }
    }
  }
  d->s.nedges = nedges;
  std::vector<int> status(nedges, -1);
  std::vector<char> off_mesh(np + 1, 0);  // NOT_AN_EDGE
  for (size_t i = 0; i < p.nbv.size(); ++i) {
    int code = p.lbcodei[i];
    if (!(code == 4 || code == 24 || code == 5 || code == 25)) continue;
    int j1 = p.nbv[i], j2 = p.ibconn[i];
    for (const Segment& seg : p.segments) {
      int t = seg.ibtype;
      if (!(t == 0 || t == 3 || t == 2 || t == 12 || t == 13 || t == 20 || t == 22 || t == 23 || t == 1 ||
            t == 11 || t == 21))
        continue;
      for (size_t q = 0; q + 1 < seg.nodes.size(); ++q) {
        int n1 = seg.nodes[q], n2 = seg.nodes[q + 1];
        if ((n1 == j1 || n1 == j2) && (n2 == j1 || n2 == j2)) off_mesh[n1] = off_mesh[n2] = 1;
      }
    }
  }
  d->niedn.clear();
  for (int i = 0; i < nedges; ++i)
    if (d->nedel[2 * (size_t)i] != 0 && d->nedel[2 * (size_t)i + 1] != 0) {
      d->niedn.push_back(i + 1);
      status[i] = 0;
    }
  std::vector<std::vector<std::pair<int, int>>> adjacency(np + 1);
  for (int i = 0; i < nedges; ++i) {
    int a = d->nedno[2 * (size_t)i], b = d->nedno[2 * (size_t)i + 1];
    adjacency[a].push_back({b, i + 1});
    adjacency[b].push_back({a, i + 1});
  }
  auto edge_of = [&](int a, int b) {
    for (auto& pr : adjacency[a])
      if (pr.first == b) return pr.second;
    return 0;
  };
  for (const auto& seg : p.open_segments)
    for (size_t q = 0; q + 1 < seg.size(); ++q) {
      int id = edge_of(seg[q], seg[q + 1]);
      if (id == 0) throw dgswem::Failure(DGSWEM_ERR_IO, "open boundary node pair is not an element edge");
      d->needn.push_back(id);
      status[id - 1] = 4;
    }
  size_t wall_seg = 0;
  for (const Segment& seg : p.segments) {
    int t = seg.ibtype;
    for (size_t q = 0; q + 1 < seg.nodes.size(); ++q) {
      int n1 = seg.nodes[q], n2 = seg.nodes[q + 1];
      if (off_mesh[n1] && off_mesh[n2]) continue;
      int id = edge_of(n1, n2);
      if (id == 0) continue;
      status[id - 1] = 1;
      if (t == 0 || t == 10 || t == 20 || t == 1 || t == 11 || t == 21) d->nledn.push_back(id);
      if (t == 2 || t == 12 || t == 22) d->nfedn.push_back(id);
      if (t == 3 || t == 13 || t == 23) d->nebsegn.push_back(id);
      if (t == 4 || t == 14 || t == 24) {
        int other = 0;
        if (wall_seg < p.backnodes.size()) {
          int b1 = p.backnodes[wall_seg].first, b2 = p.backnodes[wall_seg].second;
          for (int j = 0; j < nedges; ++j) {
            int c1 = d->nedno[2 * (size_t)j], c2 = d->nedno[2 * (size_t)j + 1];
            if ((b1 == c1 || b1 == c2) && (b2 == c1 || b2 == c2)) {
              other = j + 1;
              status[j] = 1;
            }
          }
        }
        d->nibsegn.push_back(id);
        d->nibsegn.push_back(other);
        ++wall_seg;
      }
      if (t == 30) d->nredn.push_back(id);
    }
  }
  for (int i = 0; i < nedges; ++i)
    if (status[i] < 0) d->nledn.push_back(i + 1);  // unclassified -> land
  d->nedsd.assign(2 * (size_t)nedges, 0);
  for (int i = 0; i < nedges; ++i)
    for (int side = 0; side < 2; ++side) {
      int e = d->nedel[2 * (size_t)i + side];
      if (e == 0) continue;
      for (int l = 0; l < 3; ++l)
        if (d->neled[l + 3 * (size_t)(e - 1)] == i + 1) d->nedsd[2 * (size_t)i + side] = l + 1;
    }
  dgswem_cuda_setup& s = d->s;
  s.nieds = (int)d->niedn.size();
  s.nleds = (int)d->nledn.size();
  s.needs = (int)d->needn.size();
  s.nfeds = (int)d->nfedn.size();
  s.nreds = (int)d->nredn.size();
  s.nebseg = (int)d->nebsegn.size();
  s.nibseg = (int)d->nibsegn.size() / 2;
}

// HB modes, per-element forcing, initial wet/dry, boundary forcing tables
void build_element_data(dgswem_deck* d, const Fort15& p) {
  dgswem_cuda_setup& s = d->s;
  const int ne = s.ne, dofh = s.dofh;
  auto NM = [&](int e, int v) { return d->nm[e + (size_t)ne * v] - 1; };
  d->hb.assign((size_t)dofh * ne, 0.0);
  d->cori_el.resize(ne);
  d->fric_el.resize(ne);
  std::vector<double> corif(s.np, p.cori);
  if (p.ncor == 1)
    for (int n = 0; n < s.np; ++n) corif[n] = 2.0 * 7.29212e-5 * std::sin(d->sfea[n]);
  for (int e = 0; e < ne; ++e) {
    int a = NM(e, 0), b = NM(e, 1), c = NM(e, 2);
    const double* DP = d->dp.data();
    d->hb[(size_t)dofh * e + 0] = 1.0 / 3.0 * (DP[a] + DP[b] + DP[c]);
    d->hb[(size_t)dofh * e + 1] = -(1.0 / 6.0 * (DP[a] + DP[b])) + 1.0 / 3.0 * DP[c];
    d->hb[(size_t)dofh * e + 2] = -(0.5 * DP[a]) + 0.5 * DP[b];
    d->cori_el[e] = (corif[a] + corif[b] + corif[c]) / 3.0;
    d->fric_el[e] = (s.cf + s.cf + s.cf) / 3.0;
  }
  d->ze.assign((size_t)dofh * ne, 0.0);
  d->qx.assign((size_t)dofh * ne, 0.0);
  d->qy.assign((size_t)dofh * ne, 0.0);
  d->wdflg.assign(ne, 1);
  if (s.nolifa == 2) {  // prep_DG.F:1214-1274 (cold start)
    for (int e = 0; e < ne; ++e) {
      double* z = &d->ze[(size_t)dofh * e];
      double v[3];
      for (int k = 0; k < 3; ++k) {
        double dpn = d->dp[NM(e, k)];
        v[k] = z[0];
        if (dpn < s.h0) v[k] = std::max(v[k], s.h0 - dpn);
      }
      double mean = (v[0] + v[1] + v[2]) / 3.0;
      if (mean != z[0]) {
        if (z[0] > mean) {
          for (int k = 1; k < dofh; ++k) z[k] = 0.0;
        } else {
          z[0] = mean;
          z[1] = -(1.0 / 6.0 * (v[0] + v[1])) + 1.0 / 3.0 * v[2];
          z[2] = -(0.5 * v[0]) + 0.5 * v[1];
        }
        d->wdflg[e] = 0;
      }
    }
  }
  // EMO_DG(NBFR,NEEDS,2) in the order of the open-boundary edges
  const int nb = std::max(p.nbfr, 1), needs = s.needs;
  d->emo_dg.assign((size_t)nb * needs * 2, 0.0);
  d->efa_dg.assign((size_t)nb * needs * 2, 0.0);
  for (int f = 0; f < p.nbfr; ++f) {
    int edge = 0, node = 0;
    for (const auto& seg : p.open_segments) {
      for (size_t q = 0; q + 1 < seg.size(); ++q, ++edge, ++node)
        for (int ipt = 0; ipt < 2; ++ipt) {
          size_t at = f + (size_t)nb * (edge + (size_t)needs * ipt);
          d->emo_dg[at] = p.emo[f][node + ipt];
          d->efa_dg[at] = p.efa[f][node + ipt];
        }
      ++node;
    }
  }
  const int nq = std::max(p.nffr, 1), nfeds = s.nfeds;
  d->qnam_dg.assign((size_t)nq * nfeds * 2, 0.0);
  d->qnph_dg.assign((size_t)nq * nfeds * 2, 0.0);
  for (int f = 0; f < p.nffr; ++f) {
    int edge = 0, node = 0;
    for (const Segment& seg : p.segments) {
      int t = seg.ibtype;
      if (!(t == 2 || t == 12 || t == 22)) continue;
      for (size_t q = 0; q + 1 < seg.nodes.size(); ++q, ++edge, ++node)
        if (edge < nfeds && node + 1 < (int)p.qnam[f].size())
          for (int ipt = 0; ipt < 2; ++ipt) {
            size_t at = f + (size_t)nq * (edge + (size_t)nfeds * ipt);
            d->qnam_dg[at] = p.qnam[f][node + ipt];
            d->qnph_dg[at] = p.qnph[f][node + ipt];
          }
      ++node;
    }
  }
}

}  // namespace

// DG hot start (prep_DG.F:1403-1445, MODAL_IC = 2): Hot_start.263 (PH, then
// ZE(K,J) one per record), Hot_start.264 (PH PH, then QX(K,J) QY(K,J)) and
// Hot_start.214 (ITHS ..., then HB(K,J) WDFLG(J)), records in the order J
// = 1..NE, K = 1..DOFH, read list-directed (the items a record needs, the
// rest of it skipped; D exponents accepted).  The modes replace the cold
// start's ZE/QX/QY, HB and WDFLG.
namespace {
std::vector<std::vector<double>> hot_records(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw dgswem::Failure(DGSWEM_ERR_IO, "cannot open " + path);
  std::vector<std::vector<double>> recs;
  std::string line;
  while (std::getline(in, line)) {
    for (char& c : line)
      if (c == ',') c = ' ';
      else if (c == 'D' || c == 'd') c = 'E';
    std::vector<double> v;
    const char* p = line.c_str();
    char* end = nullptr;
    for (;;) {
      const double x = std::strtod(p, &end);
      if (end == p) break;
      v.push_back(x);
      p = end;
    }
    if (!v.empty()) recs.push_back(std::move(v));
  }
  return recs;
}
}  // namespace

static void read_hotstart(const std::string& root, dgswem_deck* d) {
  const dgswem_cuda_setup& s = d->s;
  const size_t ne = (size_t)s.ne, dofh = (size_t)s.dofh, n = ne * dofh;
  auto r263 = hot_records(root + "/Hot_start.263");
  auto r264 = hot_records(root + "/Hot_start.264");
  auto r214 = hot_records(root + "/Hot_start.214");
  if (r263.size() < n + 1 || r264.size() < n + 1 || r214.size() < n + 1)
    throw dgswem::Failure(DGSWEM_ERR_IO, "DG hot start files hold fewer records than NE x DOFH");
  if ((int)r263[0][0] != d->ph || r264[0].size() < 2 || (int)r264[0][0] != d->ph)
    throw dgswem::Failure(DGSWEM_ERR_IO, "INCONSISTENCY IN P -- CHECK INPUT FILES (DG hot start)");
  d->hot_it = (int)r214[0][0];
  for (size_t i = 0; i < n; ++i) {
    const auto &a = r263[i + 1], &b = r264[i + 1], &c = r214[i + 1];
    if (b.size() < 2 || c.size() < 2) throw dgswem::Failure(DGSWEM_ERR_IO, "short DG hot start record");
    d->ze[i] = a[0];
    d->qx[i] = b[0];
    d->qy[i] = b[1];
    d->hb[i] = c[0];
    d->wdflg[i / dofh] = (int)c[1];
  }
}

extern "C" int dgswem_deck_open(const char* dir, dgswem_deck** out) {
  return dgswem::guarded([&]() {
    if (!dir || !out) throw dgswem::Failure(DGSWEM_ERR_ARG, "null argument");
    std::unique_ptr<dgswem_deck> d(new dgswem_deck());
    Fort15 p;
    std::string root(dir);
    read_fort_dg(root, d.get());
    read_fort14_15(root, d.get(), &p);
    if (d->pl != d->ph) throw dgswem::Failure(DGSWEM_ERR_ARG, "p-adaptivity (pl != ph) is not supported");
    if (d->ph != 1 && d->ph != 2) throw dgswem::Failure(DGSWEM_ERR_ARG, "only p = 1 and p = 2 are supported");
    if (d->ph == 2 && (d->s.slopeflag != 0 || d->s.nolifa >= 2))
      throw dgswem::Failure(DGSWEM_ERR_ARG, "the slope limiter and wetting/drying are p = 1 only, as in the reference");
    if (d->modal_ic != 0 && d->modal_ic != 2)
      throw dgswem::Failure(DGSWEM_ERR_ARG, "modal_ic must be 0 (cold start) or 2 (DG hot start)");
    if (d->artdif != 0 || d->sedflag != 0)
      throw dgswem::Failure(DGSWEM_ERR_ARG, "artificial diffusion / sediment are not on this path");
    d->s.dofh = (d->ph + 1) * (d->ph + 2) / 2;
    rk_tables(d.get());
    d->s.nrk = d->rk_stage;
    build_edges(d.get(), p);
    build_element_data(d.get(), p);
    if (d->modal_ic == 2) read_hotstart(root, d.get());
    dgswem_cuda_setup& s = d->s;
    s.atvd = d->atvd.data();
    s.btvd = d->btvd.data();
    s.dtvd = d->dtvd.data();
    s.nm = d->nm.data();
    s.x = d->x.data();
    s.y = d->y.data();
    s.dp = d->dp.data();
    s.nedno = d->nedno.data();
    s.nedel = d->nedel.data();
    s.nedsd = d->nedsd.data();
    s.neled = d->neled.data();
    s.niedn = d->niedn.data();
    s.nledn = d->nledn.data();
    s.needn = d->needn.data();
    s.nfedn = d->nfedn.data();
    s.nredn = d->nredn.data();
    s.nebsegn = d->nebsegn.data();
    s.nibsegn = d->nibsegn.data();
    s.hb = d->hb.data();
    s.cori_el = d->cori_el.data();
    s.fric_el = d->fric_el.data();
    s.manning = d->manning.empty() ? nullptr : d->manning.data();
    s.ze = d->ze.data();
    s.qx = d->qx.data();
    s.qy = d->qy.data();
    s.wdflg = d->wdflg.data();
    s.nbfr = (int)d->amig.size();
    s.amig = d->amig.data();
    s.ff = d->ff.data();
    s.face = d->face.data();
    s.per = d->per.data();
    s.emo_dg = d->emo_dg.data();
    s.efa_dg = d->efa_dg.data();
    s.nffr = (int)d->famig.size();
    s.famig = d->famig.data();
    s.fff = d->fff.data();
    s.fface = d->fface.data();
    s.fper = d->fper.data();
    s.qnam_dg = d->qnam_dg.data();
    s.qnph_dg = d->qnph_dg.data();
    s.ebht = d->ebht.data();
    s.ebcfsp = d->ebcfsp.data();
    s.ibht = d->ibht.data();
    s.ibcfsb = d->ibcfsb.data();
    s.ibcfsp = d->ibcfsp.data();
    *out = d.release();
  });
}

extern "C" const dgswem_cuda_setup* dgswem_deck_setup(const dgswem_deck* d) { return d ? &d->s : nullptr; }

extern "C" int dgswem_deck_int(const dgswem_deck* d, const char* key, int* value) {
  return dgswem::guarded([&]() {
    if (!d || !key || !value) throw dgswem::Failure(DGSWEM_ERR_ARG, "null argument");
    std::string k(key);
    if (k == "nt") *value = d->nt;
    else if (k == "nspoolge") *value = d->nspoolge;
    else if (k == "ntcysge") *value = d->ntcysge;
    else if (k == "ntcyfge") *value = d->ntcyfge;
    else if (k == "noutge") *value = d->noutge;
    else if (k == "dghot") *value = d->dghot;
    else if (k == "dghotspool") *value = d->dghotspool;
    else if (k == "modal_ic") *value = d->modal_ic;
    else if (k == "hotstart_it") *value = d->hot_it;
    else throw dgswem::Failure(DGSWEM_ERR_ARG, "unknown deck key " + k);
  });
}

extern "C" void dgswem_deck_close(dgswem_deck* d) { delete d; }

// ---- ensembles -------------------------------------------------------------
// One setup holding n independent meshes side by side (no shared nodes, so no
// edge joins two instances): every per-node, per-element, per-edge and
// per-boundary-edge array is concatenated and its ids offset by the preceding
// instances' counts.  A handle created from it advances all instances in
// each kernel launch.  What the kernels read as one value for the whole mesh
// (time step, RK tables, physics switches and constants, tidal and flow
// constituents) must be the same in every instance; per-instance forcing
// lives in the per-edge amplitudes (EMO_DG/EFA_DG, QNAM_DG/QNPH_DG), the
// nodal Manning n and the nodal met fields.  No counterpart in the reference
// (one mesh per run there).
namespace {

template <class T>
void append_offset(std::vector<T>& dst, const T* src, size_t n, T off, bool keep_zero) {
  for (size_t i = 0; i < n; ++i) dst.push_back(keep_zero && src[i] == 0 ? 0 : src[i] + off);
}

template <class T>
void append(std::vector<T>& dst, const T* src, size_t n) {
  if (n) dst.insert(dst.end(), src, src + n);
}

bool same(const double* a, const double* b, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!(a[i] == b[i])) return false;
  return true;
}

void check_compatible(const dgswem_cuda_setup& a, const dgswem_cuda_setup& b, int i) {
  auto fail = [&](const char* what) {
    throw dgswem::Failure(DGSWEM_ERR_ARG, "ensemble member " + std::to_string(i) + ": " + what +
                                              " differs from member 0 (it is one value for the whole ensemble)");
  };
  if (a.dofh != b.dofh || a.nrk != b.nrk) fail("DOFH / RK stages");
  if (a.ics != b.ics || a.nolifa != b.nolifa || a.iflinbf != b.iflinbf || a.ifhybf != b.ifhybf ||
      a.ifnlfa != b.ifnlfa || a.nramp != b.nramp || a.nws != b.nws || a.rainfall != b.rainfall ||
      a.slopeflag != b.slopeflag || a.load_manning != b.load_manning)
    fail("a physics switch");
  const double sa[] = {a.nleq, a.leq, a.g, a.h0, a.dtdp, a.statim, a.dramp, a.cf, a.hbreak, a.ftheta, a.fgamma, a.sfea0};
  const double sb[] = {b.nleq, b.leq, b.g, b.h0, b.dtdp, b.statim, b.dramp, b.cf, b.hbreak, b.ftheta, b.fgamma, b.sfea0};
  if (!same(sa, sb, sizeof(sa) / sizeof(sa[0]))) fail("a physics constant or the time step");
  const size_t nn = (size_t)a.nrk * a.nrk;
  if (!same(a.atvd, b.atvd, nn) || !same(a.btvd, b.btvd, nn) || !same(a.dtvd, b.dtvd, a.nrk)) fail("the RK tables");
  if (a.nbfr != b.nbfr || !same(a.amig, b.amig, a.nbfr) || !same(a.ff, b.ff, a.nbfr) ||
      !same(a.face, b.face, a.nbfr) || !same(a.per, b.per, a.nbfr))
    fail("the tidal constituents");
  if (a.nffr != b.nffr || !same(a.famig, b.famig, a.nffr) || !same(a.fff, b.fff, a.nffr) ||
      !same(a.fface, b.fface, a.nffr) || !same(a.fper, b.fper, a.nffr))
    fail("the flow constituents");
}

// per-boundary-edge harmonic table X(NF, NEDGE, 2) of every member into the
// merged X(NF, sum NEDGE, 2)
void merge_harmonic(std::vector<double>& dst, const std::vector<const dgswem_cuda_setup*>& p, int nf,
                    int dgswem_cuda_setup::*count, const double* dgswem_cuda_setup::*arr) {
  const int nb = std::max(nf, 1);
  size_t total = 0;
  for (auto* s : p) total += (size_t)(s->*count);
  dst.assign((size_t)nb * total * 2, 0.0);
  size_t off = 0;
  for (auto* s : p) {
    const int ned = s->*count;
    const double* src = s->*arr;
    if (src && nf > 0)
      for (int f = 0; f < nf; ++f)
        for (int e = 0; e < ned; ++e)
          for (int ipt = 0; ipt < 2; ++ipt)
            dst[f + (size_t)nb * ((off + e) + total * ipt)] = src[f + (size_t)nb * (e + (size_t)ned * ipt)];
    off += ned;
  }
}

}  // namespace

extern "C" int dgswem_deck_merge(const dgswem_cuda_setup* const* parts, int n, dgswem_deck** out) {
  return dgswem::guarded([&]() {
    if (!parts || !out || n < 1) throw dgswem::Failure(DGSWEM_ERR_ARG, "null argument or empty ensemble");
    *out = nullptr;
    std::vector<const dgswem_cuda_setup*> p(parts, parts + n);
    for (int i = 0; i < n; ++i) {
      if (!p[i]) throw dgswem::Failure(DGSWEM_ERR_ARG, "null ensemble member");
      if (i) check_compatible(*p[0], *p[i], i);
    }
    std::unique_ptr<dgswem_deck> d(new dgswem_deck());
    const dgswem_cuda_setup& s0 = *p[0];
    dgswem_cuda_setup& s = d->s;
    s = s0;  // switches, constants, counts of constituents
    long long ne = 0, np = 0, ned = 0;
    s.nieds = s.nleds = s.needs = s.nfeds = s.nreds = s.nebseg = s.nibseg = 0;
    for (auto* m : p) {
      ne += m->ne; np += m->np; ned += m->nedges;
      s.nieds += m->nieds; s.nleds += m->nleds; s.needs += m->needs; s.nfeds += m->nfeds;
      s.nreds += m->nreds; s.nebseg += m->nebseg; s.nibseg += m->nibseg;
    }
    if (ne > INT32_MAX / 3 || np > INT32_MAX || ned > INT32_MAX / 2)
      throw dgswem::Failure(DGSWEM_ERR_ARG, "ensemble exceeds 32-bit element / node / edge ids");
    s.ne = (int)ne; s.np = (int)np; s.nedges = (int)ned;
    d->nm.assign(3 * (size_t)ne, 0);
    d->neled.assign(3 * (size_t)ne, 0);
    int eoff = 0, noff = 0, edoff = 0;
    for (auto* m : p) {
      for (int v = 0; v < 3; ++v)
        for (int e = 0; e < m->ne; ++e) d->nm[(size_t)(eoff + e) + (size_t)ne * v] = m->nm[e + (size_t)m->ne * v] + noff;
      for (size_t i = 0; i < 3 * (size_t)m->ne; ++i)
        d->neled[3 * (size_t)eoff + i] = m->neled[i] == 0 ? 0 : m->neled[i] + edoff;
      append(d->x, m->x, m->np);
      append(d->y, m->y, m->np);
      append(d->dp, m->dp, m->np);
      if (s.load_manning) append(d->manning, m->manning, m->np);
      append_offset(d->nedno, m->nedno, 2 * (size_t)m->nedges, noff, true);
      append_offset(d->nedel, m->nedel, 2 * (size_t)m->nedges, eoff, true);
      append(d->nedsd, m->nedsd, 2 * (size_t)m->nedges);
      append_offset(d->niedn, m->niedn, m->nieds, edoff, false);
      append_offset(d->nledn, m->nledn, m->nleds, edoff, false);
      append_offset(d->needn, m->needn, m->needs, edoff, false);
      append_offset(d->nfedn, m->nfedn, m->nfeds, edoff, false);
      append_offset(d->nredn, m->nredn, m->nreds, edoff, false);
      append_offset(d->nebsegn, m->nebsegn, m->nebseg, edoff, false);
      append_offset(d->nibsegn, m->nibsegn, 2 * (size_t)m->nibseg, edoff, true);
      append(d->hb, m->hb, (size_t)s0.dofh * m->ne);
      append(d->cori_el, m->cori_el, m->ne);
      append(d->fric_el, m->fric_el, m->ne);
      append(d->ze, m->ze, (size_t)s0.dofh * m->ne);
      append(d->qx, m->qx, (size_t)s0.dofh * m->ne);
      append(d->qy, m->qy, (size_t)s0.dofh * m->ne);
      append(d->wdflg, m->wdflg, m->ne);
      append(d->ebht, m->ebht, m->nebseg);
      append(d->ebcfsp, m->ebcfsp, m->nebseg);
      append(d->ibht, m->ibht, m->nibseg);
      append(d->ibcfsb, m->ibcfsb, m->nibseg);
      append(d->ibcfsp, m->ibcfsp, m->nibseg);
      eoff += m->ne; noff += m->np; edoff += m->nedges;
    }
    merge_harmonic(d->emo_dg, p, s0.nbfr, &dgswem_cuda_setup::needs, &dgswem_cuda_setup::emo_dg);
    merge_harmonic(d->efa_dg, p, s0.nbfr, &dgswem_cuda_setup::needs, &dgswem_cuda_setup::efa_dg);
    merge_harmonic(d->qnam_dg, p, s0.nffr, &dgswem_cuda_setup::nfeds, &dgswem_cuda_setup::qnam_dg);
    merge_harmonic(d->qnph_dg, p, s0.nffr, &dgswem_cuda_setup::nfeds, &dgswem_cuda_setup::qnph_dg);
    d->atvd.assign(s0.atvd, s0.atvd + (size_t)s0.nrk * s0.nrk);
    d->btvd.assign(s0.btvd, s0.btvd + (size_t)s0.nrk * s0.nrk);
    d->dtvd.assign(s0.dtvd, s0.dtvd + s0.nrk);
    d->amig.assign(s0.amig, s0.amig + s0.nbfr);
    d->ff.assign(s0.ff, s0.ff + s0.nbfr);
    d->face.assign(s0.face, s0.face + s0.nbfr);
    d->per.assign(s0.per, s0.per + s0.nbfr);
    d->famig.assign(s0.famig, s0.famig + s0.nffr);
    d->fff.assign(s0.fff, s0.fff + s0.nffr);
    d->fface.assign(s0.fface, s0.fface + s0.nffr);
    d->fper.assign(s0.fper, s0.fper + s0.nffr);
    s.atvd = d->atvd.data(); s.btvd = d->btvd.data(); s.dtvd = d->dtvd.data();
    s.nm = d->nm.data(); s.x = d->x.data(); s.y = d->y.data(); s.dp = d->dp.data();
    s.nedno = d->nedno.data(); s.nedel = d->nedel.data(); s.nedsd = d->nedsd.data(); s.neled = d->neled.data();
    s.niedn = d->niedn.data(); s.nledn = d->nledn.data(); s.needn = d->needn.data(); s.nfedn = d->nfedn.data();
    s.nredn = d->nredn.data(); s.nebsegn = d->nebsegn.data(); s.nibsegn = d->nibsegn.data();
    s.hb = d->hb.data(); s.cori_el = d->cori_el.data(); s.fric_el = d->fric_el.data();
    s.manning = d->manning.empty() ? nullptr : d->manning.data();
    s.ze = d->ze.data(); s.qx = d->qx.data(); s.qy = d->qy.data(); s.wdflg = d->wdflg.data();
    s.amig = d->amig.data(); s.ff = d->ff.data(); s.face = d->face.data(); s.per = d->per.data();
    s.emo_dg = d->emo_dg.data(); s.efa_dg = d->efa_dg.data();
    s.famig = d->famig.data(); s.fff = d->fff.data(); s.fface = d->fface.data(); s.fper = d->fper.data();
    s.qnam_dg = d->qnam_dg.data(); s.qnph_dg = d->qnph_dg.data();
    s.ebht = d->ebht.data(); s.ebcfsp = d->ebcfsp.data();
    s.ibht = d->ibht.data(); s.ibcfsb = d->ibcfsb.data(); s.ibcfsp = d->ibcfsp.data();
    *out = d.release();
  });
}

// ---- NWS = 1 meteorological forcing file (fort.22) -------------------------
// met_forcing.F:49-66: every call of MET_FORCING -- once per RK stage,
// DG_hydro_timestep.F:104 -- reads NP records `READ(22,*) NHG, WSX2(II),
// WSY2(II), PR2(II)`, II = 1..NP, in input node order.  Each list-directed
// READ starts a new record and takes four values, continuing on the
// following lines if a line holds fewer; values after the fourth on its
// last line are skipped.  Separators are blanks, tabs and commas; a D
// exponent (1.0D-3) reads as E.
struct dgswem_met_reader {
  std::FILE* f = nullptr;
  std::string path;
  int np = 0;
  long line = 0;  // lines consumed
  long calls = 0; // blocks of NP records read
  std::vector<char> buf;
  ~dgswem_met_reader() {
    if (f) std::fclose(f);
  }
  // the next line into buf (without its end of line); false at end of file
  bool next_line() {
    buf.clear();
    int c;
    bool any = false;
    while ((c = std::fgetc(f)) != EOF) {
      any = true;
      if (c == '\n') break;
      buf.push_back((char)c);
    }
    if (!any) return false;
    ++line;
    if (!buf.empty() && buf.back() == '\r') buf.pop_back();
    buf.push_back(0);
    return true;
  }
  // one list-directed READ of four values
  void read_record(double v[4]) {
    int got = 0;
    while (got < 4) {
      if (!next_line())
        throw dgswem::Failure(DGSWEM_ERR_IO, path + ": end of file in record block " + std::to_string(calls + 1) +
                                                 " (NP = " + std::to_string(np) + " records per MET_FORCING call)");
      char* p = buf.data();
      while (got < 4) {
        while (*p == ' ' || *p == '\t' || *p == ',') ++p;
        if (!*p) break;
        char* q = p;
        while (*q && *q != ' ' && *q != '\t' && *q != ',') {
          if (*q == 'D' || *q == 'd') *q = 'E';
          ++q;
        }
        const char end = *q;
        *q = 0;
        char* stop = nullptr;
        const double x = std::strtod(p, &stop);
        if (stop == p || *stop)
          throw dgswem::Failure(DGSWEM_ERR_IO, path + ":" + std::to_string(line) + ": not a number: " + p);
        v[got++] = x;
        *q = end;
        p = q;
      }
    }
  }
};

extern "C" int dgswem_met_reader_open(const char* path, int np, dgswem_met_reader** out) {
  return dgswem::guarded([&]() {
    if (!path || !out || np <= 0) throw dgswem::Failure(DGSWEM_ERR_ARG, "bad arguments");
    std::unique_ptr<dgswem_met_reader> r(new dgswem_met_reader());
    r->path = path;
    r->np = np;
    r->f = std::fopen(path, "rb");
    if (!r->f) throw dgswem::Failure(DGSWEM_ERR_IO, std::string("cannot open ") + path);
    *out = r.release();
  });
}

void dgswem::met_read_block(dgswem_met_reader* r, double* wsx2, double* wsy2, double* pr2) {
  if (!r || !wsx2 || !wsy2 || !pr2) throw dgswem::Failure(DGSWEM_ERR_ARG, "null argument");
  double v[4];
  for (int i = 0; i < r->np; ++i) {
    r->read_record(v);  // NHG (the node number) is read and not used, as in the reference
    wsx2[i] = v[1];
    wsy2[i] = v[2];
    pr2[i] = v[3];
  }
  ++r->calls;
}

extern "C" int dgswem_met_reader_next(dgswem_met_reader* r, double* wsx2, double* wsy2, double* pr2) {
  return dgswem::guarded([&]() { dgswem::met_read_block(r, wsx2, wsy2, pr2); });
}

extern "C" long dgswem_met_reader_calls(const dgswem_met_reader* r) { return r ? r->calls : -1; }

extern "C" void dgswem_met_reader_close(dgswem_met_reader* r) { delete r; }
