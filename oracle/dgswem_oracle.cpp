/*
 * dgswem_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never shipped).
 *
 * CPU FP64 restatement of the DG-SWEM explicit DG hydro time step and of the
 * setup it depends on.  Every routine names the reference file:line it
 * follows (paths relative to the reference project root).  Loops keep the
 * reference's evaluation order so rounding follows the reference build (it is
 * compiled with -ffp-contract=off; the reference's own gfortran -march=native
 * build may contract a*b+c, so agreement with its golden files is at print
 * precision, not bitwise).
 *
 * Scope (the parity path): p=1; p=2 generalised as in the p-generic boundary
 * code -- the interior-edge sums run over every mode, where the reference's
 * internal_edge_hydro.F:306-318,337-345 sum modes 1-3 only (its p=2 defect,
 * which makes the higher modes unstable) -- and checked by its convergence
 * order, not pinned to the reference; LLF flux (numerical_flux.F:750-1022, the flux the
 * reference compiles with _FLUX=2), SSP-RK (RKSSP), SLOPELIMITER5, WETDRY,
 * ocean/land/flow/radiation/external-barrier/internal-barrier edges, NWS=0/1,
 * rainfall=0/1, ICS=1/2, NOLIBF=0/1/2, Manning n from fort.13.
 *
 * Deviation stated up front: node stars (limiter node pass, modal2nodal) are
 * taken in element order instead of the reference's angle-sorted ELETAB walk
 * (prep_DG.F:297-336).  min/max over a set does not depend on the order; the
 * modal2nodal area-weighted sum differs only in rounding.
 */
#include "dgswem_oracle.h"

#include <quadmath.h>

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

static const double PI = 3.141592653589793;       // global.F:72
static const double DEG2RAD = PI / 180.0;         // global.F:73
static const double BARMIN = 0.01;                // global.F:89
static const double R_EARTH = 6378206.4;          // dgswem.F:617

struct Err : std::runtime_error { using std::runtime_error::runtime_error; };

// DEPTH**(1.D0/3.D0) of the Manning friction (rhs_dg_hydro.F), correctly
// rounded.  The reference's gfortran build calls the C library's pow, whose
// result is within 0.52 ulp of x^c (c = RN(1/3)) but not always the nearest
// double (about 1 evaluation in 1,200 of depths in [1e-3, 1e3] is one ulp
// off); the oracle takes the nearest double, which pins the rounding of this
// expression independently of any math library.  Method (Ziv's strategy):
// d = pow(x, c); its relative error e is measured in x87 extended precision
// (64-bit significand) from d^3 = x^(3c) (1 + 3e), x^(3c) = x (1 - 2^-54 ln x);
// the nearest of d and its two neighbours is returned unless x^c lies within
// 2^-60 relative of a midpoint, where the quadruple-precision pow decides.
static_assert(LDBL_MANT_DIG == 64, "x87 extended precision expected");
static double pow_third_cr(double x) {
  const double d = std::pow(x, 1.0 / 3.0);
  if (!(x > 0.0) || !(d < INFINITY) || !(d > 0.0)) return d;
  const long double D = d;
  const long double target = (long double)x * (1.0L - 0x1p-54L * (long double)std::log(x));
  const long double e = ((D * D * D) / target - 1.0L) / 3.0L;  // d = x^c (1 + e)
  const double up = std::nextafter(d, INFINITY), dn = std::nextafter(d, -INFINITY);
  // d - x^c = e x^c ~ e d; midpoints at d + (up - d)/2 and d - (d - dn)/2
  const long double dev = e * D;
  const long double hu = 0.5L * ((long double)up - D), hd = 0.5L * (D - (long double)dn);
  const long double tol = D * 0x1p-60L;
  if (std::fabs(dev + hu) <= tol || std::fabs(dev - hd) <= tol) return (double)powq((__float128)x, (__float128)(1.0 / 3.0));
  if (dev < -hu) return up;   // x^c above the upper midpoint
  if (dev > hd) return dn;    // x^c below the lower midpoint
  return d;
}

// ---------------------------------------------------------------- readers --
// Fortran list-directed input: a READ takes the next record and, if it holds
// fewer values than asked for, continues on the following records.
struct FortFile {
  std::vector<std::string> lines;
  size_t pos = 0;
  std::string name;
  void open(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw Err("cannot open " + path);
    name = path;
    std::string s;
    while (std::getline(f, s)) {
      if (!s.empty() && s.back() == '\r') s.pop_back();
      lines.push_back(s);
    }
  }
  bool eof() const { return pos >= lines.size(); }
  std::string line() {
    if (pos >= lines.size()) throw Err("unexpected end of " + name);
    return lines[pos++];
  }
  static void split(const std::string& s, std::vector<std::string>& out) {
    std::string cur;
    for (char c : s) {
      if (c == '/') break;  // list-directed terminator
      if (std::isspace((unsigned char)c) || c == ',') {
        if (!cur.empty()) { out.push_back(cur); cur.clear(); }
      } else {
        cur.push_back(c);
      }
    }
    if (!cur.empty()) out.push_back(cur);
  }
  std::vector<std::string> values(size_t n) {
    std::vector<std::string> v;
    while (v.size() < n) {
      std::vector<std::string> t;
      split(line(), t);
      for (auto& x : t) { if (v.size() < n) v.push_back(x); }
    }
    return v;
  }
  static double to_real(std::string s) {
    for (auto& c : s) if (c == 'd' || c == 'D') c = 'E';
    char* end = nullptr;
    double v = std::strtod(s.c_str(), &end);
    if (end == s.c_str()) throw Err("bad real '" + s + "'");
    return v;
  }
  static long to_int(const std::string& s) {
    char* end = nullptr;
    long v = std::strtol(s.c_str(), &end, 10);
    if (end == s.c_str()) throw Err("bad integer '" + s + "'");
    return v;
  }
  double real() { return to_real(values(1)[0]); }
  long integer() { return to_int(values(1)[0]); }
};

// ------------------------------------------------------------------ model --
struct Model {
  // fort.dg (read_fort_dg.F90:449-484 keywords)
  int pl = 1, ph = 1, fluxtype = 2, rk_stage = 2, rk_order = 2, modal_ic = 0;
  int slopeflag = 5, rainfall = 0, artdif = 0, sedflag = 0;
  // fort.15
  int NFOVER = 0, ICS = 1, IM = 0, NOLIBF = 0, NOLIFA = 0, NSTARTDRY = 0;
  int NOLICA = 0, NOLICAT = 0, NWP = 0, NCOR = 0, NTIP = 0, NWS = 0, NRS = 0;
  int NRAMP = 0;
  double G = 9.81, TAU0 = 0, DTDP = 1, STATIM = 0, REFTIM = 0, RNDAY = 0;
  double DRAMP = 1, DRAMPExtFlux = 1, H0 = 0, SLAM0 = 0, SFEA0 = 0;
  double TAU = 0, CF = 0, HBREAK = 1, FTHETA = 1, FGAMMA = 1, CORI = 0;
  int NTIF = 0, NBFR = 0;
  std::vector<double> AMIG, FF, FACE, PER;
  int NOUTGE = 0, NSPOOLGE = 0, NT = 0, NTCYSGE = 0, NTCYFGE = 0;
  double TOUTSGE = 0, TOUTFGE = 0;
  bool LoadManningsN = false;
  std::vector<double> ManningsN;
  // derived flags (dgswem.F:131-170)
  int IFLINBF = 1, IFHYBF = 0, IFNLFA = 0;
  double NLEQ = 0, LEQ = 1, NLEQG = 0, FG_L = 0;
  std::string RUNDES, RUNID, AGRID;

  // fort.14 mesh (0-based)
  int NE = 0, NP = 0;
  std::vector<double> X, Y, DP, SLAM, SFEA, SFAC, AREAS;
  std::vector<int> NM;  // NM[3*e + v], 0-based node ids
  // open boundaries
  int NOPE = 0, NETA = 0;
  std::vector<std::vector<int>> NBDV;
  std::vector<std::vector<double>> EMO, EFA;  // [freq][neta]
  // land boundaries; NBVV[k] holds indices 0..NVELL+1 as the reference's
  // NBVV(K,0:NVELL+1)
  int NBOU = 0;
  std::vector<int> NVELL, SEGTYPE;
  std::vector<std::vector<int>> NBVV;
  // global boundary-node lists NBV/IBCONN/LBCODEI (read_input.F:2531-2660)
  std::vector<int> NBV, IBCONN, LBCODEI;
  std::vector<double> EBHT, EBCFSP, IBHT, IBCFSB, IBCFSP;
  std::vector<std::pair<int, int>> BACKNODES;
  // flow boundaries
  int NFFR = 0;
  std::vector<double> FAMIG, FFF, FFACE, FPER;
  std::vector<std::vector<double>> QNAM, QNPH;  // [freq][flow node]

  // RK (prep_DG.F:1551-2078)
  int NRK = 0;
  std::vector<double> ATVD, BTVD, DTVD;  // ATVD[(i-1)*NRK + (j-1)]

  // DG tables
  int dofh = 3, NAGP = 3, NEGP = 3;
  std::vector<double> XAGP, YAGP, WAGP, XEGP, WEGP;
  std::vector<double> PHI_AREA, DRPHI, DSPHI;  // [k*NAGP + i]
  std::vector<double> PHI_EDGE;                // [(led*NEGP + i)*dofh + k]
  std::vector<double> PHI_CORNER;              // [v*dofh + k]
  std::vector<double> M_INV;
  std::vector<double> PSI1, PSI2, PSI3;
  double DRPSI[3] = {-0.5, 0.5, 0.0}, DSPSI[3] = {-0.5, 0.0, 0.5};
  double C13 = 1.0 / 3.0, C16 = 1.0 / 6.0;

  // edges (create_edge_data.F)
  int NEDGES = 0;
  std::vector<int> NEDNO, NEDEL, NELED, NEDSD;  // NEDNO[2*ed+s]; NELED[3*e+l]
  std::vector<int> NIEDN, NLEDN, NEEDN, NFEDN, NREDN, NEBSEGN, NIBSEGN, NIBEDN;
  std::vector<int> ELEM_EDGE;  // [3*e + slot], -1 if empty
  std::vector<double> XLEN, COSNX, SINNX;

  // per element
  std::vector<double> DRDX, DSDX, DRDY, DSDY, CORI_EL, FRIC_EL, DPE_MIN;
  std::vector<double> BATH, DBATHDX, DBATHDY, SFAC_ELEM;  // [e*NAGP + i]
  std::vector<double> XFAC, YFAC, SRFAC;  // [(e*dofh + k)*NAGP + i]
  std::vector<double> BATHED, SFACED;     // [(e*3 + led)*NEGP + i]
  std::vector<double> EDGEQ;              // [(led*NEGP + i)*dofh + k]
  std::vector<double> DP_NODE;            // [3*e + v]
  std::vector<double> EMO_DG, EFA_DG;     // [(f*NEEDS + l)*2 + ipt]
  std::vector<double> QNAM_DG, QNPH_DG;
  std::vector<double> CORIF, FRIC;

  // state: ZE[(s*NE + e)*dofh + k], s = 0..NRK  (reference stage s+1)
  std::vector<double> ZE, QX, QY, RHS_ZE, RHS_QX, RHS_QY, HB;
  std::vector<double> ze_edge, qx_edge, qy_edge;  // [(e*3+slot)*dofh + k]
  std::vector<int> WDFLG, NODECODE;
  std::vector<double> WSX2, WSY2, PR2, WSX_BASE, WSY_BASE, PR_BASE;
  // NWS = 1: unit 22 (fort.22 of the deck), read at every MET_FORCING call
  // (met_forcing.F:49-66) unless the fields are given with orc_set_met
  std::FILE* F22 = nullptr;
  std::string F22_path;
  void met_read_fort22();
  ~Model() { if (F22) std::fclose(F22); }
  // node star in element order: star[star_ptr[n] .. star_ptr[n+1])
  std::vector<int> star_ptr, star;

  // ------------------------------------------------------------ helpers --
  double& ze(int s, int e, int k) { return ZE[((size_t)s * NE + e) * dofh + k]; }
  double& qx(int s, int e, int k) { return QX[((size_t)s * NE + e) * dofh + k]; }
  double& qy(int s, int e, int k) { return QY[((size_t)s * NE + e) * dofh + k]; }
  double& rze(int s, int e, int k) { return RHS_ZE[((size_t)s * NE + e) * dofh + k]; }
  double& rqx(int s, int e, int k) { return RHS_QX[((size_t)s * NE + e) * dofh + k]; }
  double& rqy(int s, int e, int k) { return RHS_QY[((size_t)s * NE + e) * dofh + k]; }
  double& hb(int e, int k) { return HB[(size_t)e * dofh + k]; }
  double phi_edge(int k, int i, int led) const { return PHI_EDGE[((size_t)led * NEGP + i) * dofh + k]; }
  double edgeq(int k, int i, int led) const { return EDGEQ[((size_t)led * NEGP + i) * dofh + k]; }
  double phi_corner(int k, int v) const { return PHI_CORNER[(size_t)v * dofh + k]; }
  double atvd(int i, int j) const { return ATVD[(size_t)(i - 1) * NRK + (j - 1)]; }
  double btvd(int i, int j) const { return BTVD[(size_t)(i - 1) * NRK + (j - 1)]; }

  void read_fort_dg(const std::string& dir);
  void read_input(const std::string& dir);
  void read_fort13(const std::string& dir);
  void rk_time();
  void create_edge_data();
  void prep_dg();
  void step(int it);
  void modal2nodal(double* eta2, double* uu2, double* vv2) const;

  // stage routines (irk is 1-based as in the reference)
  int IRK = 1;
  double TIMEDG = 0, RAMPDG = 1;
  void ocean_edges();
  void land_edges();
  void flow_edges();
  void radiation_edges();
  void ebarrier_edges();
  void ibarrier_edges();
  void internal_edges();
  void add_internal_flux();
  void rhs_dg_hydro();
  void ssp_update();
  void slopelimiter5();
  void wetdry();
};

// numerical_flux.F:750-914 (LLF).  NLEQ/LEQ/FG_L are the model's; G is the
// argument (the dry-side calls pass 0).
static inline void llf_flux(const Model& m, double ze_in, double ze_ex, double qx_in,
                            double qx_ex, double qy_in, double qy_ex, double hb_in,
                            double hb_ex, double sfac_in, double sfac_ex, double nx,
                            double ny, double G, double out[3]) {
  const double NLEQ = m.NLEQ, LEQ = m.LEQ, FG_L = m.FG_L;
  double NLEQG = G * NLEQ;
  double J1 = ze_ex - ze_in, J2 = qx_ex - qx_in, J3 = qy_ex - qy_in;
  double HT_IN = ze_in * NLEQ + hb_in;
  double F1_NL = NLEQ + LEQ * hb_in;
  double FX1_IN = qx_in * F1_NL * sfac_in;
  double FY1_IN = qy_in * F1_NL;
  double FU_NL = NLEQ * qx_in, FV_NL = NLEQ * qy_in, FG_NL = NLEQG * ze_in;
  double FH_NL = 1.0 / (NLEQ * HT_IN + LEQ);
  double U_IN = qx_in * FH_NL, V_IN = qy_in * FH_NL;
  double HUU = FU_NL * U_IN, HVV = FV_NL * V_IN, HUV = FU_NL * V_IN;
  double GH2 = FG_NL * (0.5 * ze_in + hb_in) + FG_L * ze_in;
  double FX2_IN = (HUU + GH2) * sfac_in, FY2_IN = HUV;
  double FX3_IN = HUV * sfac_in, FY3_IN = HVV + GH2;

  double HT_EX = ze_ex * NLEQ + hb_ex;
  F1_NL = NLEQ + LEQ * hb_ex;
  double FX1_EX = qx_ex * F1_NL * sfac_ex;
  double FY1_EX = qy_ex * F1_NL;
  FU_NL = NLEQ * qx_ex; FV_NL = NLEQ * qy_ex; FG_NL = NLEQG * ze_ex;
  FH_NL = 1.0 / (NLEQ * HT_EX + LEQ);
  double U_EX = qx_ex * FH_NL, V_EX = qy_ex * FH_NL;
  HUU = FU_NL * U_EX; HVV = FV_NL * V_EX; HUV = FU_NL * V_EX;
  GH2 = FG_NL * (0.5 * ze_ex + hb_ex) + FG_L * ze_ex;
  double FX2_EX = (HUU + GH2) * sfac_ex, FY2_EX = HUV;
  double FX3_EX = HUV * sfac_ex, FY3_EX = HVV + GH2;

  double F1_AVG = 0.5 * ((FX1_IN + FX1_EX) * nx + (FY1_IN + FY1_EX) * ny);
  double F2_AVG = 0.5 * ((FX2_IN + FX2_EX) * nx + (FY2_IN + FY2_EX) * ny);
  double F3_AVG = 0.5 * ((FX3_IN + FX3_EX) * nx + (FY3_IN + FY3_EX) * ny);

  double UN_IN = (U_IN * nx + V_IN * ny) * NLEQ;
  double C_IN = std::sqrt(G * HT_IN * (ny * ny + (nx * sfac_in) * (nx * sfac_in)));
  double e1 = std::fabs(UN_IN + C_IN), e2 = std::fabs(UN_IN), e3 = std::fabs(UN_IN - C_IN);
  double UN_EX = (U_EX * nx + V_EX * ny) * NLEQ;
  double C_EX = std::sqrt(G * HT_EX * (ny * ny + (nx * sfac_ex) * (nx * sfac_ex)));
  double e4 = std::fabs(UN_EX + C_EX), e5 = std::fabs(UN_EX), e6 = std::fabs(UN_EX - C_EX);
  double EIGMAX = std::max(std::max(std::max(e1, e2), std::max(e3, e4)), std::max(e5, e6));

  double NX2 = NLEQ + LEQ * nx * nx, NY2 = NLEQ + LEQ * ny * ny, NXY = nx * ny;
  out[0] = F1_AVG - 0.5 * EIGMAX * J1;
  out[1] = F2_AVG - 0.5 * EIGMAX * (J2 * NX2 + LEQ * J3 * NXY);
  out[2] = F3_AVG - 0.5 * EIGMAX * (J3 * NY2 + LEQ * J2 * NXY);
}

// ------------------------------------------------------ fort.dg reading --
// read_fort_dg.F90:186-300 (keyword) and :73-185 (fixed); detection
// read_input.F:191-201.
void Model::read_fort_dg(const std::string& dir) {
  FortFile f;
  f.open(dir + "/fort.dg");
  std::string first;
  {
    std::vector<std::string> t;
    FortFile::split(f.lines.empty() ? std::string() : f.lines[0], t);
    first = t.empty() ? std::string() : t[0];
  }
  if (!first.empty() && first[0] == '1') {
    f.integer();                          // DGSWE
    f.values(2);                          // padapt, pflag
    f.values(2);                          // gflag, diorism
    auto p = f.values(3);
    pl = (int)FortFile::to_int(p[0]); ph = (int)FortFile::to_int(p[1]);
    f.values(1); f.values(1); f.values(3);  // slimit, plimit, k ks L
    fluxtype = (int)f.integer();
    auto r = f.values(2);
    rk_stage = (int)FortFile::to_int(r[0]); rk_order = (int)FortFile::to_int(r[1]);
    f.values(1);                          // DG_TO_CG
    modal_ic = (int)f.integer();
    f.values(2);                          // DGHOT, DGHOTSPOOL
    slopeflag = (int)f.integer();
    auto s = f.values(4);
    sedflag = (int)FortFile::to_int(s[0]);
    f.values(1); f.values(1);
    auto a = f.values(5);
    artdif = (int)FortFile::to_int(a[0]);
    return;
  }
  // keyword format; defaults from FORT_DG_SETUP
  pl = 1; ph = 1; fluxtype = 1; rk_stage = 2; rk_order = 2; modal_ic = 0;
  slopeflag = 5; rainfall = 0; artdif = 0; sedflag = 0;
  for (auto& raw : f.lines) {
    size_t b = raw.find_first_not_of(" \t");
    if (b == std::string::npos) continue;
    std::string line = raw.substr(b);
    if (line[0] == '!') continue;
    size_t eq = line.find('=');
    if (eq == std::string::npos) continue;
    std::string key = line.substr(0, eq);
    while (!key.empty() && std::isspace((unsigned char)key.back())) key.pop_back();
    size_t ex = line.find('!');
    std::string val = (ex != std::string::npos && ex > eq) ? line.substr(eq + 1, ex - eq - 1)
                                                           : line.substr(eq + 1);
    std::vector<std::string> t;
    FortFile::split(val, t);
    if (t.empty()) continue;
    auto I = [&]() { return (int)FortFile::to_int(t[0]); };
    if (key == "pl") pl = I();
    else if (key == "ph") ph = I();
    else if (key == "fluxtype") fluxtype = I();
    else if (key == "rk_stage") rk_stage = I();
    else if (key == "rk_order") rk_order = I();
    else if (key == "modal_ic") modal_ic = I();
    else if (key == "slopeflag") slopeflag = I();
    else if (key == "rainfall") rainfall = I();
    else if (key == "artdif") artdif = I();
    else if (key == "sedflag") sedflag = I();
  }
}

// ----------------------------------------------------- fort.13 (Manning) --
// nodalattr.F:295-700 (only mannings_n_at_sea_floor is loaded)
void Model::read_fort13(const std::string& dir) {
  FortFile f;
  f.open(dir + "/fort.13");
  f.line();
  long nn = f.integer();
  if (nn != NP) throw Err("fort.13 node count mismatch");
  long nattr = f.integer();
  std::vector<std::string> names;
  std::vector<double> defs;
  for (long k = 0; k < nattr; ++k) {
    std::string name = f.line();
    size_t b = name.find_first_not_of(" \t"), e = name.find_last_not_of(" \t");
    name = (b == std::string::npos) ? "" : name.substr(b, e - b + 1);
    f.line();                        // units
    long nv = f.integer();
    auto d = f.values((size_t)nv);
    names.push_back(name);
    defs.push_back(FortFile::to_real(d[0]));
  }
  for (long k = 0; k < nattr; ++k) {
    std::string name = f.line();
    size_t b = name.find_first_not_of(" \t"), e = name.find_last_not_of(" \t");
    name = (b == std::string::npos) ? "" : name.substr(b, e - b + 1);
    long cnt = f.integer();
    size_t idx = std::find(names.begin(), names.end(), name) - names.begin();
    bool want = (name == "mannings_n_at_sea_floor") && LoadManningsN;
    if (want) ManningsN.assign(NP, idx < defs.size() ? defs[idx] : 0.0);
    for (long i = 0; i < cnt; ++i) {
      std::string ln = f.line();
      if (want) {
        std::vector<std::string> t;
        FortFile::split(ln, t);
        long node = FortFile::to_int(t[0]);
        ManningsN[node - 1] = FortFile::to_real(t[1]);
      }
    }
  }
  if (LoadManningsN && ManningsN.empty()) throw Err("fort.13 lacks mannings_n_at_sea_floor");
}

// --------------------------------------------------- fort.15 / fort.14 ----
// read_input.F:209-2970 (positional subset this path needs)
void Model::read_input(const std::string& dir) {
  FortFile f15, f14;
  f15.open(dir + "/fort.15");
  f14.open(dir + "/fort.14");
  RUNDES = f15.line();
  RUNID = f15.line();
  NFOVER = (int)f15.integer();
  f15.integer();  // NABOUT
  f15.integer();  // NSCREEN
  long IHOT = f15.integer();
  if (IHOT != 0) throw Err("IHOT != 0 (ADCIRC hot start) is outside the DG path");
  ICS = (int)f15.integer();
  IM = (int)f15.integer();
  NOLIBF = (int)f15.integer();
  NOLIFA = (int)f15.integer();
  NSTARTDRY = 0;
  if (NOLIFA == 3) { NOLIFA = 2; NSTARTDRY = 1; }
  NOLICA = (int)f15.integer();
  NOLICAT = (int)f15.integer();
  NWP = (int)f15.integer();
  for (int k = 0; k < NWP; ++k) {  // nodalattr.F:352-390
    std::string a = f15.line();
    if (a.find("mannings_n_at_sea_floor") != std::string::npos) LoadManningsN = true;
  }
  NCOR = (int)f15.integer();
  NTIP = (int)f15.integer();
  if (NTIP != 0) throw Err("NTIP != 0 (tidal potential) is not on this path");
  NWS = (int)f15.integer();
  NRS = 0;
  if (std::abs(NWS / 100) >= 1) { NRS = 1; NWS = (std::abs(NWS) - 100) * (NWS / std::abs(NWS)); }
  if (std::abs(NWS / 100) >= 2) { NRS = 1; NWS = (std::abs(NWS) - 200) * (NWS / std::abs(NWS)); }
  if (NWS != 0 && NWS != 1) throw Err("only NWS=0/1 are on this path");
  if (NRS != 0) throw Err("NRS != 0 (radiation stress) is not on this path");
  NRAMP = (int)f15.integer();
  G = f15.real();
  TAU0 = f15.real();
  DTDP = f15.real();
  STATIM = f15.real();
  REFTIM = f15.real();
  RNDAY = f15.real();
  NT = (int)(RNDAY * (86400.0 / DTDP) + 0.5);
  if (NRAMP == 0 || NRAMP == 1) {
    DRAMP = f15.real();
    DRAMPExtFlux = DRAMP;
  } else if (NRAMP >= 2 && NRAMP <= 7) {
    auto v = f15.values((size_t)(NRAMP + 1 >= 3 ? NRAMP + 1 : 3));
    DRAMP = FortFile::to_real(v[0]);
    DRAMPExtFlux = FortFile::to_real(v[1]);
  } else {
    throw Err("bad NRAMP");
  }
  f15.values(3);  // A00 B00 C00
  if (NOLIFA != 2) H0 = f15.real();
  else H0 = FortFile::to_real(f15.values(4)[0]);
  AGRID = f14.line();
  {
    auto v = f14.values(2);
    NE = (int)FortFile::to_int(v[0]);
    NP = (int)FortFile::to_int(v[1]);
  }
  {
    auto v = f15.values(2);
    SLAM0 = FortFile::to_real(v[0]) * DEG2RAD;
    SFEA0 = FortFile::to_real(v[1]) * DEG2RAD;
  }
  X.assign(NP, 0); Y.assign(NP, 0); DP.assign(NP, 0); SLAM.assign(NP, 0); SFEA.assign(NP, 0);
  for (int i = 0; i < NP; ++i) {
    auto v = f14.values(4);
    int j = (int)FortFile::to_int(v[0]) - 1;
    if (j < 0 || j >= NP) throw Err("bad node number in fort.14");
    if (ICS == 1) {
      X[j] = FortFile::to_real(v[1]); Y[j] = FortFile::to_real(v[2]);
      SLAM[j] = SLAM0 + X[j] / (R_EARTH * std::cos(SFEA0));  // INVCP dgswem.F:631
      SFEA[j] = Y[j] / R_EARTH;
    } else {
      SLAM[j] = DEG2RAD * FortFile::to_real(v[1]);
      SFEA[j] = DEG2RAD * FortFile::to_real(v[2]);
      X[j] = R_EARTH * (SLAM[j] - SLAM0) * std::cos(SFEA0);  // CPP dgswem.F:614
      Y[j] = SFEA[j] * R_EARTH;
    }
    DP[j] = FortFile::to_real(v[3]);
  }
  SFAC.assign(NP, 1.0);
  if (ICS == 2)
    for (int i = 0; i < NP; ++i) SFAC[i] = std::cos(SFEA0) / std::cos(SFEA[i]);
  if (NOLIFA == 0 || NOLIFA == 1)  // read_input.F:1356
    for (int i = 0; i < NP; ++i) if (DP[i] < H0) DP[i] = H0;
  NM.assign(3 * (size_t)NE, 0);
  AREAS.assign(NE, 0);
  for (int i = 0; i < NE; ++i) {
    auto v = f14.values(5);
    int j = (int)FortFile::to_int(v[0]) - 1;
    if (j < 0 || j >= NE) throw Err("bad element number in fort.14");
    for (int a = 0; a < 3; ++a) NM[3 * j + a] = (int)FortFile::to_int(v[2 + a]) - 1;
    double X1 = X[NM[3 * j]], X2 = X[NM[3 * j + 1]], X3 = X[NM[3 * j + 2]];
    double Y1 = Y[NM[3 * j]], Y2 = Y[NM[3 * j + 1]], Y3 = Y[NM[3 * j + 2]];
    AREAS[j] = (X1 - X3) * (Y2 - Y3) + (X3 - X2) * (Y1 - Y3);  // read_input.F:1406
    if (AREAS[j] < 0.0) throw Err("element " + std::to_string(j + 1) + " is clockwise");
  }
  if (NSTARTDRY == 1) throw Err("NOLIFA=3 (fort.12 start-dry) is not supported");
  // friction (read_input.F:1668-1679)
  HBREAK = 1.0; FTHETA = 1.0; FGAMMA = 1.0;
  if (NOLIBF == 0) TAU = f15.real();
  CF = TAU;
  if (NOLIBF == 1) CF = f15.real();
  if (NOLIBF == 2) {
    auto v = f15.values(4);
    CF = FortFile::to_real(v[0]); HBREAK = FortFile::to_real(v[1]);
    FTHETA = FortFile::to_real(v[2]); FGAMMA = FortFile::to_real(v[3]);
  }
  FRIC.assign(NP, CF);
  if (IM == 10) f15.values(2); else f15.values(1);  // ESLM (ESLC)
  if (NWP > 0) read_fort13(dir);
  CORI = f15.real();
  CORIF.assign(NP, CORI);
  if (NCOR == 1)
    for (int i = 0; i < NP; ++i) CORIF[i] = 2.0 * 7.29212e-5 * std::sin(SFEA[i]);
  NTIF = (int)f15.integer();
  for (int i = 0; i < NTIF; ++i) { f15.line(); f15.values(5); }
  NBFR = (int)f15.integer();
  AMIG.assign(NBFR, 0); FF.assign(NBFR, 0); FACE.assign(NBFR, 0); PER.assign(NBFR, 0);
  for (int i = 0; i < NBFR; ++i) {
    f15.line();
    auto v = f15.values(3);
    AMIG[i] = FortFile::to_real(v[0]); FF[i] = FortFile::to_real(v[1]);
    FACE[i] = FortFile::to_real(v[2]) * DEG2RAD;
    PER[i] = (AMIG[i] == 0.0) ? 0.0 : 2.0 * PI / AMIG[i];
  }
  // open boundaries (read_input.F:2015-2060)
  NOPE = (int)f14.integer();
  NETA = (int)f14.integer();
  NBDV.assign(NOPE, {});
  int jnmm = 0;
  for (int k = 0; k < NOPE; ++k) {
    int nv = (int)f14.integer();
    for (int i = 0; i < nv; ++i) NBDV[k].push_back((int)f14.integer() - 1);
    jnmm += nv;
  }
  if (jnmm != NETA) {
    if (NFOVER == 1) NETA = jnmm; else throw Err("NETA mismatch in fort.14");
  }
  if (NBFR == 0 && NOPE > 0) throw Err("non-periodic elevation boundaries (fort.19) are not supported");
  EMO.assign(NBFR, std::vector<double>(NETA, 0.0));
  EFA.assign(NBFR, std::vector<double>(NETA, 0.0));
  for (int i = 0; i < NBFR; ++i) {
    f15.line();
    for (int j = 0; j < NETA; ++j) {
      auto v = f15.values(2);
      EMO[i][j] = FortFile::to_real(v[0]);
      EFA[i][j] = FortFile::to_real(v[1]) * DEG2RAD;
    }
  }
  f15.values(1);  // ANGINN
  // land boundaries (read_input.F:2144-2690)
  NBOU = (int)f14.integer();
  f14.integer();  // NVEL
  NVELL.assign(NBOU, 0); SEGTYPE.assign(NBOU, 0); NBVV.assign(NBOU, {});
  bool nfluxf = false;
  for (int k = 0; k < NBOU; ++k) {
    auto v = f14.values(2);
    int nvell = (int)FortFile::to_int(v[0]);
    int ib = (int)FortFile::to_int(v[1]);
    SEGTYPE[k] = ib;
    bool ext_bar = (ib == 3 || ib == 13 || ib == 23);
    bool int_bar = (ib == 4 || ib == 24);
    bool pipe = (ib == 5 || ib == 25);
    bool ok = ib == 0 || ib == 10 || ib == 20 || ib == 1 || ib == 11 || ib == 21 || ib == 2 ||
              ib == 12 || ib == 22 || ext_bar || int_bar || ib == 30;
    if (!ok) throw Err("boundary type " + std::to_string(ib) + " is not supported");
    (void)pipe;
    if (ib == 2 || ib == 12 || ib == 22) nfluxf = true;
    std::vector<int> nb(nvell), ibc(nvell);
    std::vector<double> ht(nvell), cfsb(nvell), cfsp(nvell);
    for (int i = 0; i < nvell; ++i) {
      if (ext_bar) {
        auto t = f14.values(3);
        nb[i] = (int)FortFile::to_int(t[0]) - 1;
        ht[i] = FortFile::to_real(t[1]); cfsp[i] = FortFile::to_real(t[2]);
      } else if (int_bar) {
        auto t = f14.values(5);
        nb[i] = (int)FortFile::to_int(t[0]) - 1; ibc[i] = (int)FortFile::to_int(t[1]) - 1;
        ht[i] = FortFile::to_real(t[2]); cfsb[i] = FortFile::to_real(t[3]);
        cfsp[i] = FortFile::to_real(t[4]);
      } else {
        nb[i] = (int)f14.integer() - 1;
      }
    }
    int nprbi = int_bar ? 2 : 1;
    for (int ip = 1; ip <= nprbi; ++ip) {
      if (ip == 2) {  // second pass: swap sides and reverse (read_input.F:2447-2470)
        std::vector<int> nb2(nvell), ibc2(nvell);
        std::vector<double> ht2(nvell), cb2(nvell), cp2(nvell);
        for (int i = 0; i < nvell; ++i) {
          nb2[i] = ibc[nvell - 1 - i]; ibc2[i] = nb[nvell - 1 - i];
          ht2[i] = ht[nvell - 1 - i]; cb2[i] = cfsb[nvell - 1 - i]; cp2[i] = cfsp[nvell - 1 - i];
        }
        nb = nb2; ibc = ibc2; ht = ht2; cfsb = cb2; cfsp = cp2;
      }
      // NBVV(K,0:NVELL+1) with island closing (read_input.F:2489-2500)
      std::vector<int> bv(nb);
      if (ib == 1 || ib == 11 || ib == 21)
        if (bv.back() != bv.front()) bv.push_back(bv.front());
      int nv2 = (int)bv.size();
      std::vector<int> full(nv2 + 2);
      for (int i = 0; i < nv2; ++i) full[i + 1] = bv[i];
      full[0] = bv[0];
      if (bv[nv2 - 1] == bv[0]) full[0] = bv[nv2 - 2];
      full[nv2 + 1] = bv[nv2 - 1];
      NBVV[k] = full;
      NVELL[k] = nv2;
      for (int i = 0; i < nv2; ++i) {
        NBV.push_back(bv[i]);
        LBCODEI.push_back(ib);
        IBCONN.push_back((int_bar && i < nvell) ? ibc[i] : -1);
      }
    }
    if (ext_bar)
      for (int i = 0; i + 1 < nvell; ++i) {
        EBHT.push_back(0.5 * (ht[i] + ht[i + 1]));
        EBCFSP.push_back(0.5 * (cfsp[i] + cfsp[i + 1]));
      }
    if (int_bar)
      for (int i = 0; i + 1 < nvell; ++i) {
        IBHT.push_back(0.5 * (ht[i] + ht[i + 1]));
        IBCFSB.push_back(0.5 * (cfsb[i] + cfsb[i + 1]));
        IBCFSP.push_back(0.5 * (cfsp[i] + cfsp[i + 1]));
        BACKNODES.push_back({ibc[i], ibc[i + 1]});
      }
  }
  // flow boundaries (read_input.F:2971-3045, DGSWE=1 compact indexing)
  if (nfluxf) {
    NFFR = (int)f15.integer();
    if (NFFR == 0) throw Err("non-periodic flux boundaries (fort.20) are not supported");
    FAMIG.assign(NFFR, 0); FFF.assign(NFFR, 0); FFACE.assign(NFFR, 0); FPER.assign(NFFR, 0);
    for (int i = 0; i < NFFR; ++i) {
      f15.line();
      auto v = f15.values(3);
      FAMIG[i] = FortFile::to_real(v[0]); FFF[i] = FortFile::to_real(v[1]);
      FFACE[i] = FortFile::to_real(v[2]) * DEG2RAD;
      FPER[i] = (FAMIG[i] == 0.0) ? 0.0 : 2.0 * PI / FAMIG[i];
    }
    int nflow = 0;
    for (size_t j = 0; j < LBCODEI.size(); ++j)
      if (LBCODEI[j] == 2 || LBCODEI[j] == 12 || LBCODEI[j] == 22) ++nflow;
    QNAM.assign(NFFR, std::vector<double>(nflow, 0.0));
    QNPH.assign(NFFR, std::vector<double>(nflow, 0.0));
    for (int i = 0; i < NFFR; ++i) {
      f15.line();
      for (int j = 0; j < nflow; ++j) {
        auto v = f15.values(2);
        QNAM[i][j] = FortFile::to_real(v[0]);
        QNPH[i][j] = FortFile::to_real(v[1]) * DEG2RAD;
      }
    }
  }
  // output control (read_input.F:3169-3935)
  auto skip_stations = [&](bool) {
    long n = f15.integer();
    for (long i = 0; i < n; ++i) f15.values(2);
  };
  f15.values(4); skip_stations(true);            // NOUTE + stations
  f15.values(4); skip_stations(true);            // NOUTV + stations
  if (IM == 10) { f15.values(4); skip_stations(true); }
  if (NWS != 0) { f15.values(4); skip_stations(true); }
  {
    auto v = f15.values(4);
    NOUTGE = (int)FortFile::to_int(v[0]);
    TOUTSGE = FortFile::to_real(v[1]);
    TOUTFGE = FortFile::to_real(v[2]);
    NSPOOLGE = (int)FortFile::to_int(v[3]);
    NTCYSGE = (int)((TOUTSGE - STATIM) * (86400.0 / DTDP) + 0.5);
    NTCYFGE = (int)((TOUTFGE - STATIM) * (86400.0 / DTDP) + 0.5);
    if (NTCYFGE > NT) NTCYFGE = NT;
  }
  // nonlinear flags (dgswem.F:131-170)
  if (NOLIBF == 0) { IFLINBF = 1; IFHYBF = 0; }
  if (NOLIBF == 1) { IFLINBF = 0; IFHYBF = 0; }
  if (NOLIBF == 2) { IFLINBF = 0; IFHYBF = 1; }
  IFNLFA = (NOLIFA == 0) ? 0 : 1;
  if (NOLICA == 0) { NLEQ = 0.0; LEQ = 1.0; } else { NLEQ = 1.0; LEQ = 0.0; }
  if (NOLICAT == 0) { NLEQ = 0.0; LEQ = 1.0; } else { NLEQ = 1.0; LEQ = 0.0; }
  NLEQG = NLEQ * G;
  FG_L = LEQ * G;
}

// ------------------------------------------------------------- RK_TIME ----
// prep_DG.F:1551-1990
void Model::rk_time() {
  NRK = rk_stage;
  if (NRK < 1 || NRK > 8) throw Err("bad rk_stage");
  ATVD.assign((size_t)NRK * NRK, 0.0);
  BTVD.assign((size_t)NRK * NRK, 0.0);
  std::vector<double> CTVD((size_t)NRK * NRK, 0.0);
  DTVD.assign(NRK, 0.0);
  auto A = [&](int i, int j) -> double& { return ATVD[(size_t)(i - 1) * NRK + (j - 1)]; };
  auto B = [&](int i, int j) -> double& { return BTVD[(size_t)(i - 1) * NRK + (j - 1)]; };
  auto C = [&](int i, int j) -> double& { return CTVD[(size_t)(i - 1) * NRK + (j - 1)]; };
  if (rk_stage == 1 && rk_order == 1) {
    A(1, 1) = 1.0; B(1, 1) = 1.0;
  } else if (rk_order == 2) {
    if (rk_stage == 3) {
      A(1, 1) = 1.0; A(2, 1) = 0.087353119859156; A(3, 1) = 0.344956917166841;
      A(2, 2) = 0.912646880140844; A(3, 3) = 0.655043082833159;
      B(1, 1) = 0.528005024856522; B(3, 1) = 0.022826837460491;
      B(2, 2) = 0.481882138633993; B(3, 3) = 0.345866039233415;
    } else if (rk_stage == 4) {
      A(1, 1) = 1.0; A(2, 1) = 0.394806441339829; A(3, 1) = 0.002797307087390;
      A(4, 1) = 0.252860909354373; A(2, 2) = 0.605193558660171;
      A(3, 3) = 0.997202692912610; A(4, 4) = 0.747139090645627;
      B(1, 1) = 0.406584463657504; B(3, 1) = 0.013637216641451;
      B(4, 1) = 0.016453567333598; B(2, 2) = 0.246062298456822;
      B(3, 3) = 0.405447122055692; B(4, 4) = 0.303775146447707;
    } else if (rk_stage == 5) {
      A(1, 1) = 1.0; A(2, 1) = 0.235593265061659; A(3, 1) = 0.174017972351526;
      A(4, 1) = 0.235264368870758; A(5, 1) = 0.141720372339803;
      A(2, 2) = 0.764406734938341; A(4, 2) = 0.000058643383967;
      A(5, 2) = 0.095374613155521; A(3, 3) = 0.825982027648475;
      A(5, 3) = 0.000311763705780; A(4, 4) = 0.764676987745275;
      A(5, 5) = 0.762593250798895;
      B(1, 1) = 0.324840618151514; B(3, 1) = 0.108822380501601;
      B(4, 1) = 0.054392262422093; B(5, 1) = 0.000000180291569;
      B(2, 2) = 0.248310356296551; B(4, 2) = 0.000019049753098;
      B(5, 2) = 0.030981548293401; B(3, 3) = 0.268312512443371;
      B(5, 3) = 0.000101273514903; B(4, 4) = 0.248398145385413;
      B(5, 5) = 0.247721262987686;
    } else {
      for (int I = 1; I <= NRK; ++I)
        for (int J = 0; J <= NRK - 1; ++J) {
          if (J == I - 1 && I < NRK) { A(I, J + 1) = 1.0; B(I, J + 1) = 1.0 / (NRK - 1); }
          else if (J == 0 && I == NRK) { A(I, J + 1) = 1.0 / NRK; }
          else if (J == NRK - 1 && I == NRK) { A(I, J + 1) = (NRK - 1.0) / NRK; B(I, J + 1) = 1.0 / NRK; }
        }
    }
  } else if (rk_stage == 3 && rk_order == 3) {
    A(1, 1) = 1.0; A(2, 1) = 3.0 / 4.0; A(2, 2) = 1.0 / 4.0; A(3, 1) = 1.0 / 3.0;
    A(3, 3) = 2.0 / 3.0;
    B(1, 1) = 1.0; B(2, 2) = 1.0 / 4.0; B(3, 3) = 2.0 / 3.0;
  } else {
    throw Err("unsupported rk_stage/rk_order");
  }
  for (int K = 0; K <= NRK - 1; ++K)
    for (int I = 1; I <= NRK; ++I) {
      double casum = 0.0;
      for (int L = K + 1; L <= I - 1; ++L) casum = casum + C(L, K + 1) * A(I, L + 1);
      C(I, K + 1) = B(I, K + 1) + casum;
    }
  for (int K = 1; K <= NRK - 1; ++K) {
    DTVD[K] = 0.0;
    for (int L = 0; L <= K - 1; ++L) DTVD[K] = DTVD[K] + C(K, L + 1);
  }
}

// ------------------------------------------------------ CREATE_EDGE_DATA --
// create_edge_data.F:31-635, count_edges.cpp:326-349
void Model::create_edge_data() {
  std::vector<std::vector<int>> ndel(NP);
  for (int e = 0; e < NE; ++e)
    for (int a = 0; a < 3; ++a) ndel[NM[3 * e + a]].push_back(e);
  NELED.assign(3 * (size_t)NE, -1);
  std::vector<char> edflg(3 * (size_t)NE, 0);
  NEDNO.clear(); NEDEL.clear();
  NEDGES = 0;
  for (int iel = 0; iel < NE; ++iel) {
    int n1 = NM[3 * iel], n2 = NM[3 * iel + 1], n3 = NM[3 * iel + 2];
    int led[2][3] = {{n2, n3, n1}, {n3, n1, n2}};
    for (int ied = 0; ied < 3; ++ied) {
      if (edflg[3 * iel + ied]) continue;
      int i1 = led[0][ied], i2 = led[1][ied];
      int id = NEDGES++;
      NELED[3 * iel + ied] = id;
      NEDNO.push_back(i1); NEDNO.push_back(i2);
      NEDEL.push_back(iel); NEDEL.push_back(-1);
      edflg[3 * iel + ied] = 1;
      bool done = false;
      for (int jel : ndel[i1]) {
        if (jel == iel || done) continue;
        for (int jed = 0; jed < 3; ++jed) {
          int j1 = NM[3 * jel + (jed + 1) % 3], j2 = NM[3 * jel + (jed + 2) % 3];
          if ((j1 == i1 && j2 == i2) || (j1 == i2 && j2 == i1)) {
            if (edflg[3 * jel + jed]) throw Err("possible duplicate element");
            NELED[3 * jel + jed] = id;
            NEDEL[2 * id + 1] = jel;
            edflg[3 * jel + jed] = 1;
            done = true;
            break;
          }
        }
      }
    }
  }
  std::vector<int> ncount(NEDGES, -1);
  // node pairs that are not element edges (create_edge_data.F:191-235)
  std::vector<char> not_an_edge(NP, 0);
  for (size_t ii = 0; ii < NBV.size(); ++ii) {
    int lc = LBCODEI[ii];
    if (!(lc == 4 || lc == 24 || lc == 5 || lc == 25)) continue;
    int J1 = NBV[ii], J2 = IBCONN[ii];
    for (int k = 0; k < NBOU; ++k) {
      int st = SEGTYPE[k];
      bool chk = st == 0 || st == 3 || st == 2 || st == 12 || st == 13 || st == 20 || st == 22 ||
                 st == 23 || st == 1 || st == 11 || st == 21;
      if (!chk) continue;
      for (int ied = 1; ied <= NVELL[k] - 1; ++ied) {
        int N1 = NBVV[k][ied], N2 = NBVV[k][ied + 1];
        if ((N1 == J1 || N1 == J2) && (N2 == J1 || N2 == J2)) {
          not_an_edge[N1] = 1; not_an_edge[N2] = 1;
        }
      }
    }
  }
  NIEDN.clear();
  for (int i = 0; i < NEDGES; ++i)
    if (NEDEL[2 * i] >= 0 && NEDEL[2 * i + 1] >= 0) { NIEDN.push_back(i); ncount[i] = 0; }
  // adjacency list in edge-id order (count_edges.cpp:326-349)
  std::vector<std::vector<std::pair<int, int>>> adj(NP);
  for (int i = 0; i < NEDGES; ++i) {
    adj[NEDNO[2 * i]].push_back({NEDNO[2 * i + 1], i});
    adj[NEDNO[2 * i + 1]].push_back({NEDNO[2 * i], i});
  }
  auto get_edge = [&](int a, int b) -> int {
    for (auto& p : adj[a]) if (p.first == b) return p.second;
    return -1;
  };
  NEEDN.clear();
  for (int k = 0; k < NOPE; ++k)
    for (size_t ied = 0; ied + 1 < NBDV[k].size(); ++ied) {
      int jed = get_edge(NBDV[k][ied], NBDV[k][ied + 1]);
      if (jed < 0) throw Err("error in processing open ocean boundary conditions");
      NEEDN.push_back(jed);
      ncount[jed] = 4;
    }
  NLEDN.clear(); NFEDN.clear(); NREDN.clear(); NEBSEGN.clear(); NIBSEGN.clear(); NIBEDN.clear();
  for (int k = 0; k < NBOU; ++k) {
    int st = SEGTYPE[k];
    for (int ied = 1; ied <= NVELL[k] - 1; ++ied) {
      int N1 = NBVV[k][ied], N2 = NBVV[k][ied + 1];
      if (not_an_edge[N1] && not_an_edge[N2]) continue;
      int jed = get_edge(N1, N2);
      if (jed < 0) continue;  // reported, skipped (create_edge_data.F:410-416)
      ncount[jed] = 1;
      if (st == 0 || st == 10 || st == 20 || st == 1 || st == 11 || st == 21) NLEDN.push_back(jed);
      if (st == 2 || st == 12 || st == 22) NFEDN.push_back(jed);
      if (st == 3 || st == 13 || st == 23) NEBSEGN.push_back(jed);
      if (st == 4 || st == 14 || st == 24) {
        NIBEDN.push_back(jed);
        int seg = (int)NIBSEGN.size() / 2;
        int back = -1;
        if (seg < (int)BACKNODES.size()) {
          int NN1 = BACKNODES[seg].first, NN2 = BACKNODES[seg].second;
          for (int jj = 0; jj < NEDGES; ++jj) {
            int JJ1 = NEDNO[2 * jj], JJ2 = NEDNO[2 * jj + 1];
            if ((NN1 == JJ1 || NN1 == JJ2) && (NN2 == JJ1 || NN2 == JJ2)) {
              NIBEDN.push_back(jj);
              back = jj;
              ncount[jj] = 1;
            }
          }
        }
        NIBSEGN.push_back(jed); NIBSEGN.push_back(back);
      }
      if (st == 30) NREDN.push_back(jed);
    }
  }
  for (int i = 0; i < NEDGES; ++i) {  // orphans become land (create_edge_data.F:503-524)
    int iel = NEDEL[2 * i];
    int n1 = NEDNO[2 * i], n2 = NEDNO[2 * i + 1];
    if ((n1 == NM[3 * iel + 1] && n2 == NM[3 * iel]) || (n1 == NM[3 * iel + 2] && n2 == NM[3 * iel + 1]) ||
        (n1 == NM[3 * iel] && n2 == NM[3 * iel + 2]))
      throw Err("wrong node order for an edge");
  }
  for (int i = 0; i < NEDGES; ++i)
    if (ncount[i] < 0) NLEDN.push_back(i);
  NEDSD.assign(2 * (size_t)NEDGES, -1);  // NEDSD(:,:) = 0 for a missing side
  for (int i = 0; i < NEDGES; ++i)
    for (int s = 0; s < 2; ++s) {
      int el = NEDEL[2 * i + s];
      if (el < 0) continue;
      for (int l = 0; l < 3; ++l) if (NELED[3 * el + l] == i) NEDSD[2 * i + s] = l;
    }
  ELEM_EDGE.assign(3 * (size_t)NE, -1);
  std::vector<int> cnt(NE, 0);
  for (int ged : NIEDN) {
    int a = NEDEL[2 * ged], b = NEDEL[2 * ged + 1];
    ELEM_EDGE[3 * a + cnt[a]++] = ged;
    ELEM_EDGE[3 * b + cnt[b]++] = ged;
  }
  // CALC_NORMAL (calc_normal.F:13-52)
  XLEN.assign(NEDGES, 0); COSNX.assign(NEDGES, 0); SINNX.assign(NEDGES, 0);
  for (int i = 0; i < NEDGES; ++i) {
    int n1 = NEDNO[2 * i], n2 = NEDNO[2 * i + 1];
    double dy = Y[n2] - Y[n1], dx = X[n2] - X[n1];
    XLEN[i] = std::sqrt(dy * dy + dx * dx);
    COSNX[i] = (Y[n2] - Y[n1]) / XLEN[i];
    SINNX[i] = -(X[n2] - X[n1]) / XLEN[i];
  }
}

// orthogonal_basis_v1.F:50-244 (triangle, hierarchical ordering)
static void orthogonal_basis(double X, double Y, int D, std::vector<double>& B,
                             std::vector<double>& DB1, std::vector<double>& DB2) {
  std::vector<double> PHI((D + 1) * (D + 1), 0.0), DP1((D + 1) * (D + 1), 0.0), DP2((D + 1) * (D + 1), 0.0);
  auto P_ = [&](std::vector<double>& a, int p, int q) -> double& { return a[p * (D + 1) + q]; };
  P_(PHI, 0, 0) = 1.0; P_(DP1, 0, 0) = 0.0; P_(DP2, 0, 0) = 0.0;
  if (D >= 1) {
    P_(PHI, 1, 0) = (1.0 + 2.0 * X + Y) / 2.0;
    P_(DP1, 1, 0) = 1.0;
    P_(DP2, 1, 0) = 1.0 / 2.0;
  }
  for (int P = 1; P <= D - 1; ++P) {
    double w = (1.0 - Y) / 2.0;
    double a = (2.0 * P + 1.0) / (P + 1.0), b = P / (P + 1.0);
    P_(PHI, P + 1, 0) = a * P_(PHI, 1, 0) * P_(PHI, P, 0) - b * (w * w) * P_(PHI, P - 1, 0);
    P_(DP1, P + 1, 0) = a * (P_(DP1, 1, 0) * P_(PHI, P, 0) + P_(PHI, 1, 0) * P_(DP1, P, 0)) -
                        b * (w * w) * P_(DP1, P - 1, 0);
    P_(DP2, P + 1, 0) = a * (P_(DP2, 1, 0) * P_(PHI, P, 0) + P_(PHI, 1, 0) * P_(DP2, P, 0)) -
                        b * ((Y - 1) / 2 * P_(PHI, P - 1, 0) + (w * w) * P_(DP2, P - 1, 0));
  }
  for (int P = 0; P <= D - 1; ++P) {
    double f = (1.0 + 2.0 * P + (3.0 + 2.0 * P) * Y) / 2.0;
    P_(PHI, P, 1) = P_(PHI, P, 0) * f;
    P_(DP1, P, 1) = P_(DP1, P, 0) * f;
    P_(DP2, P, 1) = P_(DP2, P, 0) * f + P_(PHI, P, 0) * (3.0 + 2.0 * P) / 2.0;
  }
  for (int Q = 1; Q <= D - 1; ++Q)
    for (int P = 0; P <= D - Q - 1; ++P) {
      double AQ = (2.0 * Q + 2.0 + 2.0 * P) * (2.0 * Q + 3.0 + 2.0 * P) / (2.0 * Q + 2.0) / (Q + 2.0 + 2.0 * P);
      double t = 2.0 * P + 1.0;
      double BQ = (t * t) * (2.0 * Q + 2.0 + 2.0 * P) / (2.0 * Q + 2.0) / (2.0 * Q + 2.0 * P + 1.0) /
                  (Q + 2.0 + 2.0 * P);
      double CQ = (Q + 2.0 * P + 1.0) * Q * (2.0 * Q + 3.0 + 2.0 * P) / (Q + 1.0) / (Q + 2.0 + 2.0 * P) /
                  (2.0 * Q + 2.0 * P + 1.0);
      P_(PHI, P, Q + 1) = (AQ * Y + BQ) * P_(PHI, P, Q) - CQ * P_(PHI, P, Q - 1);
      P_(DP1, P, Q + 1) = (AQ * Y + BQ) * P_(DP1, P, Q) - CQ * P_(DP1, P, Q - 1);
      P_(DP2, P, Q + 1) = (AQ * Y + BQ) * P_(DP2, P, Q) + AQ * P_(PHI, P, Q) - CQ * P_(DP2, P, Q - 1);
    }
  B.clear(); DB1.clear(); DB2.clear();
  for (int Q = 0; Q <= D; ++Q)
    for (int P = 0; P <= Q; ++P) {
      double b0 = P_(PHI, P, Q - P), d1 = P_(DP1, P, Q - P), d2 = P_(DP2, P, Q - P);
      if (std::fabs(b0) < 1.0e-15) b0 = 0.0;
      if (std::fabs(d1) < 1.0e-15) d1 = 0.0;
      if (std::fabs(d2) < 1.0e-15) d2 = 0.0;
      B.push_back(b0); DB1.push_back(d1); DB2.push_back(d2);
    }
}

// --------------------------------------------------------------- PREP_DG --
// prep_DG.F:25-1539
void Model::prep_dg() {
  if (pl != ph) throw Err("p-adaptivity (pl != ph) is not on this path");
  if (ph < 1 || ph > 2) throw Err("only p=1 (pinned) and p=2 (unpinned) are supported");
  if (fluxtype != 1 && fluxtype != 2 && fluxtype != 3 && fluxtype != 4) throw Err("bad fluxtype");
  if (artdif != 0) throw Err("artdif=1 (LDG diffusion) is not on this path");
  if (sedflag != 0) throw Err("sediment is not on this path");
  if (modal_ic != 0) throw Err("modal_ic != 0 is not supported by the oracle");
  if (NOLIFA >= 2 && ph != 1) throw Err("wetting/drying is p=1 in the reference");
  rk_time();
  const int p = ph;
  dofh = (p + 1) * (p + 2) / 2;
  create_edge_data();
  // area quadrature (quadrature_v1.F:245-262, 802-840)
  XAGP.clear(); YAGP.clear(); WAGP.clear();
  {
    const double V1[2] = {-1.0, -1.0}, V2[2] = {1.0, -1.0}, V3[2] = {-1.0, 1.0};
    std::vector<double> Av, Wv;
    if (p == 1) { Av = {0.1666666666666666666666666666666666}; Wv = {0.3333333333333333333333333333333333}; }
    else { Av = {0.4459484909159648863183292538830519, 0.0915762135097707434595714634022015};
           Wv = {0.2233815896780114656950070084331228, 0.1099517436553218676383263249002105}; }
    for (size_t i = 0; i < Av.size(); ++i) {
      double a = Av[i], b = Av[i], c = 1.0 - (a + b);
      double tri[3][3] = {{a, b, c}, {b, c, a}, {c, a, b}};
      for (int r = 0; r < 3; ++r) {
        XAGP.push_back(V1[0] * tri[r][0] + V2[0] * tri[r][1] + V3[0] * tri[r][2]);
        YAGP.push_back(V1[1] * tri[r][0] + V2[1] * tri[r][1] + V3[1] * tri[r][2]);
        WAGP.push_back(2.0 * Wv[i]);
      }
    }
  }
  NAGP = (int)XAGP.size();
  // edge Gauss-Lobatto (quad_rules_general.F:45-262; n=3: -1,0,1)
  NEGP = (int)std::ceil((2 * p + 3) / 2.0);
  if (NEGP == 3) {
    XEGP = {-1.0, 0.0, 1.0};
    WEGP = {2.0 / ((1.0 + 1.0) * (1.0 + 2.0)), 0.0, 0.0};
    WEGP[2] = WEGP[0];
    double x = 0.0, p0 = 1.0, p1 = x;
    double p2 = ((2.0 * 1.0 + 1.0) * x * p1 - 1.0 * p0) / (1.0 + 1.0);
    WEGP[1] = 2.0 / ((1.0 + 1.0) * (1.0 + 2.0) * p2 * p2);
  } else {
    double s = std::sqrt(1.0 / 5.0);
    XEGP = {-1.0, -s, s, 1.0};
    double nrl = 2.0;
    WEGP = {2.0 / ((nrl + 1.0) * (nrl + 2.0)), 0, 0, 0};
    WEGP[3] = WEGP[0];
    for (int m = 1; m <= 2; ++m) {
      double x = XEGP[m], pm1 = 1.0, pc = x;
      for (int q = 1; q <= 2; ++q) {
        double pn = ((2.0 * q + 1.0) * x * pc - q * pm1) / (q + 1.0);
        pm1 = pc; pc = pn;
      }
      WEGP[m] = 2.0 / ((nrl + 1.0) * (nrl + 2.0) * pc * pc);
    }
  }
  // basis at area points and corners
  PHI_AREA.assign((size_t)dofh * NAGP, 0); DRPHI.assign((size_t)dofh * NAGP, 0); DSPHI.assign((size_t)dofh * NAGP, 0);
  std::vector<double> B, D1, D2;
  for (int i = 0; i < NAGP; ++i) {
    orthogonal_basis(XAGP[i], YAGP[i], p, B, D1, D2);
    for (int k = 0; k < dofh; ++k) {
      PHI_AREA[k * NAGP + i] = B[k]; DRPHI[k * NAGP + i] = D1[k]; DSPHI[k * NAGP + i] = D2[k];
    }
  }
  PHI_CORNER.assign(3 * (size_t)dofh, 0);
  const double VX[3] = {-1.0, 1.0, -1.0}, VY[3] = {-1.0, -1.0, 1.0};
  for (int v = 0; v < 3; ++v) {
    orthogonal_basis(VX[v], VY[v], p, B, D1, D2);
    for (int k = 0; k < dofh; ++k) PHI_CORNER[v * dofh + k] = B[k];
  }
  M_INV.clear();
  for (int J = 0; J <= p; ++J)
    for (int I = 0; I <= J; ++I) {
      int JJ = J - I;
      M_INV.push_back((2.0 * I + 1.0) * (2.0 * JJ + 2.0 * I + 2.0) / 4.0);
    }
  PHI_EDGE.assign(3 * (size_t)NEGP * dofh, 0);
  for (int ii = 0; ii < 3; ++ii)
    for (int q = 0; q < NEGP; ++q) {
      double px, py;
      if (ii == 0) { px = -XEGP[q]; py = XEGP[q]; }
      else if (ii == 1) { px = -1.0; py = -XEGP[q]; }
      else { px = XEGP[q]; py = -1.0; }
      orthogonal_basis(px, py, p, B, D1, D2);
      for (int k = 0; k < dofh; ++k) PHI_EDGE[((size_t)ii * NEGP + q) * dofh + k] = B[k];
    }
  EDGEQ.assign(3 * (size_t)NEGP * dofh, 0);
  for (int l = 0; l < 3; ++l)
    for (int i = 0; i < NEGP; ++i)
      for (int k = 0; k < dofh; ++k)
        EDGEQ[((size_t)l * NEGP + i) * dofh + k] = 2.0 * M_INV[k] * phi_edge(k, i, l) * WEGP[i];
  PSI1.resize(NAGP); PSI2.resize(NAGP); PSI3.resize(NAGP);
  for (int i = 0; i < NAGP; ++i) {
    PSI1[i] = -1.0 / 2.0 * (XAGP[i] + YAGP[i]);
    PSI2[i] = 1.0 / 2.0 * (XAGP[i] + 1.0);
    PSI3[i] = 1.0 / 2.0 * (YAGP[i] + 1.0);
  }
  // state arrays
  const size_t S = (size_t)(NRK + 1) * NE * dofh;
  ZE.assign(S, 0.0); QX.assign(S, 0.0); QY.assign(S, 0.0);
  RHS_ZE.assign((size_t)NRK * NE * dofh, 0.0);
  RHS_QX = RHS_ZE; RHS_QY = RHS_ZE;
  HB.assign((size_t)NE * dofh, 0.0);
  ze_edge.assign((size_t)NE * 3 * dofh, 0.0); qx_edge = ze_edge; qy_edge = ze_edge;
  WDFLG.assign(NE, 1);
  NODECODE.assign(NP, 1);
  WSX2.assign(NP, 0.0); WSY2.assign(NP, 0.0); PR2.assign(NP, 0.0);
  // nodal -> modal bathymetry (prep_DG.F:371-377)
  std::vector<double> ydub((size_t)NE * dofh, 0.0);
  for (int j = 0; j < NE; ++j) {
    int n1 = NM[3 * j], n2 = NM[3 * j + 1], n3 = NM[3 * j + 2];
    hb(j, 0) = 1.0 / 3.0 * (DP[n1] + DP[n2] + DP[n3]);
    hb(j, 1) = -(1.0 / 6.0 * (DP[n1] + DP[n2])) + 1.0 / 3.0 * DP[n3];
    hb(j, 2) = -(0.5 * DP[n1]) + 0.5 * DP[n2];
    ydub[j * dofh + 0] = 1.0 / 3.0 * (Y[n1] + Y[n2] + Y[n3]);
    ydub[j * dofh + 1] = -(1.0 / 6.0 * (Y[n1] + Y[n2])) + 1.0 / 3.0 * Y[n3];
    ydub[j * dofh + 2] = -(0.5 * Y[n1]) + 0.5 * Y[n2];
  }
  if (p != 1) std::fill(ydub.begin(), ydub.end(), 0.0);  // YDUB(:,:,chi>1) stays 0
  DPE_MIN.resize(NE);
  for (int j = 0; j < NE; ++j)
    DPE_MIN[j] = std::min(std::min(DP[NM[3 * j]], DP[NM[3 * j + 1]]), DP[NM[3 * j + 2]]);
  // per-element tables (prep_DG.F:959-1163)
  DRDX.resize(NE); DSDX.resize(NE); DRDY.resize(NE); DSDY.resize(NE);
  CORI_EL.resize(NE); FRIC_EL.resize(NE);
  BATH.assign((size_t)NE * NAGP, 0); DBATHDX = BATH; DBATHDY = BATH; SFAC_ELEM = BATH;
  XFAC.assign((size_t)NE * dofh * NAGP, 0); YFAC = XFAC; SRFAC = XFAC;
  BATHED.assign((size_t)NE * 3 * NEGP, 0); SFACED = BATHED;
  DP_NODE.assign(3 * (size_t)NE, 0);
  for (int j = 0; j < NE; ++j) {
    int n1 = NM[3 * j], n2 = NM[3 * j + 1], n3 = NM[3 * j + 2];
    double x1 = X[n1], y1 = Y[n1], x2 = X[n2], y2 = Y[n2], x3 = X[n3], y3 = Y[n3];
    double area = (x1 - x3) * (y2 - y3) + (x3 - x2) * (y1 - y3);
    area = area * 0.5;
    DRDX[j] = 1.0 / area * (Y[n3] - Y[n1]);
    DSDX[j] = 1.0 / area * (Y[n1] - Y[n2]);
    DRDY[j] = 1.0 / area * (X[n1] - X[n3]);
    DSDY[j] = 1.0 / area * (X[n2] - X[n1]);
    CORI_EL[j] = (CORIF[n1] + CORIF[n2] + CORIF[n3]) / 3.0;
    FRIC_EL[j] = (FRIC[n1] + FRIC[n2] + FRIC[n3]) / 3.0;
    for (int i = 0; i < NAGP; ++i) {
      double bath = 0.0, dbx = 0.0, dby = 0.0, yel = 0.0;
      for (int k = 0; k < dofh; ++k) {
        double dphidx = DRPHI[k * NAGP + i] * DRDX[j] + DSPHI[k * NAGP + i] * DSDX[j];
        double dphidy = DRPHI[k * NAGP + i] * DRDY[j] + DSPHI[k * NAGP + i] * DSDY[j];
        size_t idx = ((size_t)j * dofh + k) * NAGP + i;
        XFAC[idx] = M_INV[k] * WAGP[i] * dphidx;
        YFAC[idx] = M_INV[k] * WAGP[i] * dphidy;
        SRFAC[idx] = M_INV[k] * WAGP[i] * PHI_AREA[k * NAGP + i];
        bath = bath + hb(j, k) * PHI_AREA[k * NAGP + i];
        yel = yel + ydub[j * dofh + k] * PHI_AREA[k * NAGP + i];
        dbx = dbx + hb(j, k) * dphidx;
        dby = dby + hb(j, k) * dphidy;
      }
      BATH[(size_t)j * NAGP + i] = bath;
      DBATHDX[(size_t)j * NAGP + i] = dbx;
      DBATHDY[(size_t)j * NAGP + i] = dby;
      SFAC_ELEM[(size_t)j * NAGP + i] = (ICS == 1) ? 1.0 : std::cos(SFEA0) / std::cos(yel / R_EARTH);
    }
    for (int l = 0; l < 3; ++l)
      for (int i = 0; i < NEGP; ++i) {
        double bed = 0.0, yed = 0.0;
        for (int k = 0; k < dofh; ++k) {
          bed = bed + hb(j, k) * phi_edge(k, i, l);
          yed = yed + ydub[j * dofh + k] * phi_edge(k, i, l);
        }
        BATHED[((size_t)j * 3 + l) * NEGP + i] = bed;
        SFACED[((size_t)j * 3 + l) * NEGP + i] = (ICS == 1) ? 1.0 : std::cos(SFEA0) / std::cos(yed / R_EARTH);
      }
    for (int v = 0; v < 3; ++v) DP_NODE[3 * j + v] = DP[NM[3 * j + v]];
  }
  // initial wet/dry (prep_DG.F:1214-1274; cold start, NSTARTDRY=0)
  for (int j = 0; j < NE; ++j) WDFLG[j] = 1;
  if (NOLIFA == 2) {
    for (int j = 0; j < NE; ++j) {
      double z = ze(0, j, 0);
      double Z1 = z, Z2 = z, Z3 = z;
      if (DP[NM[3 * j]] < H0) Z1 = std::max(Z1, H0 - DP[NM[3 * j]]);
      if (DP[NM[3 * j + 1]] < H0) Z2 = std::max(Z2, H0 - DP[NM[3 * j + 1]]);
      if (DP[NM[3 * j + 2]] < H0) Z3 = std::max(Z3, H0 - DP[NM[3 * j + 2]]);
      if ((Z1 + Z2 + Z3) / 3.0 != ze(0, j, 0)) {
        if (ze(0, j, 0) > (Z1 + Z2 + Z3) / 3.0) {
          for (int k = 1; k < dofh; ++k) ze(0, j, k) = 0.0;
        } else {
          ze(0, j, 0) = (Z1 + Z2 + Z3) / 3.0;
          ze(0, j, 1) = -(1.0 / 6.0 * (Z1 + Z2)) + 1.0 / 3.0 * Z3;
          ze(0, j, 2) = -(0.5 * Z1) + 0.5 * Z2;
          for (int k = 3; k < dofh; ++k) ze(0, j, k) = 0.0;
        }
        WDFLG[j] = 0;
      } else {
        WDFLG[j] = 1;
      }
    }
  }
  // ocean forcing rearranged per edge (prep_DG.F:180-205)
  int needs = (int)NEEDN.size();
  EMO_DG.assign((size_t)std::max(NBFR, 1) * needs * 2, 0.0);
  EFA_DG = EMO_DG;
  for (int f = 0; f < NBFR; ++f) {
    int ii = 0, jj = 0;
    for (int j = 0; j < NOPE; ++j) {
      for (size_t k = 0; k + 1 < NBDV[j].size(); ++k) {
        if (ii < needs) {
          EMO_DG[((size_t)f * needs + ii) * 2 + 0] = EMO[f][jj];
          EMO_DG[((size_t)f * needs + ii) * 2 + 1] = EMO[f][jj + 1];
          EFA_DG[((size_t)f * needs + ii) * 2 + 0] = EFA[f][jj];
          EFA_DG[((size_t)f * needs + ii) * 2 + 1] = EFA[f][jj + 1];
        }
        ++ii; ++jj;
      }
      ++jj;
    }
  }
  // flow forcing per edge (prep_DG.F:208-245, periodic branch)
  int nfeds = (int)NFEDN.size();
  QNAM_DG.assign((size_t)std::max(NFFR, 1) * nfeds * 2, 0.0);
  QNPH_DG = QNAM_DG;
  for (int f = 0; f < NFFR; ++f) {
    int ii = 0, jj = 0;
    for (int j = 0; j < NBOU; ++j) {
      int st = SEGTYPE[j];
      if (!(st == 2 || st == 12 || st == 22)) continue;
      for (int k = 1; k <= NVELL[j] - 1; ++k) {
        if (ii < nfeds && jj + 1 < (int)QNAM[f].size()) {
          QNAM_DG[((size_t)f * nfeds + ii) * 2 + 0] = QNAM[f][jj];
          QNAM_DG[((size_t)f * nfeds + ii) * 2 + 1] = QNAM[f][jj + 1];
          QNPH_DG[((size_t)f * nfeds + ii) * 2 + 0] = QNPH[f][jj];
          QNPH_DG[((size_t)f * nfeds + ii) * 2 + 1] = QNPH[f][jj + 1];
        }
        ++ii; ++jj;
      }
      ++jj;
    }
  }
  // node stars in element order
  star_ptr.assign(NP + 1, 0);
  for (int e = 0; e < NE; ++e) for (int a = 0; a < 3; ++a) star_ptr[NM[3 * e + a] + 1]++;
  for (int n = 0; n < NP; ++n) star_ptr[n + 1] += star_ptr[n];
  star.assign(star_ptr[NP], 0);
  {
    std::vector<int> fill(star_ptr.begin(), star_ptr.end() - 1);
    for (int e = 0; e < NE; ++e) for (int a = 0; a < 3; ++a) star[fill[NM[3 * e + a]]++] = e;
  }
}

// ------------------------------------------------------- boundary edges --
// ocean_edge_hydro.F:19-355
void Model::ocean_edges() {
  const int s = IRK - 1;
  const int needs = (int)NEEDN.size();
  for (int L = 0; L < needs; ++L) {
    int ged = NEEDN[L], led = NEDSD[2 * ged], el = NEDEL[2 * ged];
    if (WDFLG[el] == 0) continue;
    double nx = COSNX[ged], ny = SINNX[ged];
    for (int i = 0; i < NEGP; ++i) {
      double ze_in = ze(s, el, 0), qx_in = qx(s, el, 0), qy_in = qy(s, el, 0);
      double ze_ex = 0.0;
      double hb_in = BATHED[((size_t)el * 3 + led) * NEGP + i];
      double sfac_in = SFACED[((size_t)el * 3 + led) * NEGP + i];
      for (int jj = 0; jj < NBFR; ++jj) {
        double ncyc = (PER[jj] == 0.0) ? 0.0 : (double)(long long)(TIMEDG / PER[jj]);
        double argj = AMIG[jj] * (TIMEDG - ncyc * PER[jj]) + FACE[jj];
        double rff = FF[jj] * RAMPDG;
        double zg[2];
        for (int ipt = 0; ipt < 2; ++ipt) {
          double efa = EFA_DG[((size_t)jj * needs + L) * 2 + ipt];
          double emo = EMO_DG[((size_t)jj * needs + L) * 2 + ipt];
          zg[ipt] = emo * rff * std::cos(argj - efa);
        }
        double zf = 0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * XEGP[i];
        ze_ex = ze_ex + zf;
      }
      for (int k = 1; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el, k) * phi_edge(k, i, led);
        qx_in = qx_in + qx(s, el, k) * phi_edge(k, i, led);
        qy_in = qy_in + qy(s, el, k) * phi_edge(k, i, led);
      }
      double hb_ex = hb_in, sfac_ex = sfac_in;
      if (ze_ex * IFNLFA + hb_ex <= 0) ze_ex = std::fabs(hb_ex) + H0;
      double f[3];
      llf_flux(*this, ze_in, ze_ex, qx_in, qx_in, qy_in, qy_in, hb_in, hb_ex, sfac_in, sfac_ex, nx, ny, G, f);
      for (int k = 0; k < dofh; ++k) {
        double w = 2.0 * M_INV[k] / AREAS[el] * XLEN[ged] * phi_edge(k, i, led) * WEGP[i];
        rze(s, el, k) = rze(s, el, k) - w * f[0];
        rqx(s, el, k) = rqx(s, el, k) - w * f[1];
        rqy(s, el, k) = rqy(s, el, k) - w * f[2];
      }
    }
  }
}

// land_edge_hydro.F:26-311
void Model::land_edges() {
  const int s = IRK - 1;
  for (int ged : NLEDN) {
    int led = NEDSD[2 * ged], el = NEDEL[2 * ged];
    if (WDFLG[el] == 0) continue;
    double nx = COSNX[ged], ny = SINNX[ged], tx = -ny, ty = nx;
    for (int i = 0; i < NEGP; ++i) {
      double ze_in = ze(s, el, 0), qx_in = qx(s, el, 0), qy_in = qy(s, el, 0);
      double hb_in = BATHED[((size_t)el * 3 + led) * NEGP + i];
      double sfac_in = SFACED[((size_t)el * 3 + led) * NEGP + i];
      for (int k = 1; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el, k) * phi_edge(k, i, led);
        qx_in = qx_in + qx(s, el, k) * phi_edge(k, i, led);
        qy_in = qy_in + qy(s, el, k) * phi_edge(k, i, led);
      }
      double qn = qx_in * nx + qy_in * ny, qt = qx_in * tx + qy_in * ty;
      double qne = -qn, qte = qt;
      double den = 1.0 / (nx * ty - ny * tx);
      double qx_ex = (ty * qne - ny * qte) * den;
      double qy_ex = (-tx * qne + nx * qte) * den;
      double f[3];
      llf_flux(*this, ze_in, ze_in, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_in, sfac_in, sfac_in, nx, ny, G, f);
      for (int k = 0; k < dofh; ++k) {
        double w = 2.0 * M_INV[k] / AREAS[el] * XLEN[ged] * phi_edge(k, i, led) * WEGP[i];
        rze(s, el, k) = rze(s, el, k) - w * f[0];
        rqx(s, el, k) = rqx(s, el, k) - w * f[1];
        rqy(s, el, k) = rqy(s, el, k) - w * f[2];
      }
    }
  }
}

// flow_edge_hydro.F:18-333 (unpinned: no golden uses it)
void Model::flow_edges() {
  const int s = IRK - 1;
  const int nfeds = (int)NFEDN.size();
  for (int L = 0; L < nfeds; ++L) {
    int ged = NFEDN[L], led = NEDSD[2 * ged], el = NEDEL[2 * ged];
    if (WDFLG[el] == 0) continue;
    double nx = COSNX[ged], ny = SINNX[ged], tx = -ny, ty = nx;
    for (int i = 0; i < NEGP; ++i) {
      double ze_in = 0.0, qx_in = 0.0, qy_in = 0.0, qx_ex = 0.0, qy_ex = 0.0, hb_in = 0.0;
      double sfac_in = SFACED[((size_t)el * 3 + led) * NEGP + i];
      double qne = 0.0;
      for (int jj = 0; jj < NFFR; ++jj) {
        double ncyc = (FPER[jj] == 0.0) ? 0.0 : (double)(long long)(TIMEDG / FPER[jj]);
        double argj = FAMIG[jj] * (TIMEDG - ncyc * FPER[jj]) + FFACE[jj];
        double rff = FFF[jj] * RAMPDG;
        const double* qa = &QNAM_DG[((size_t)jj * nfeds + L) * 2];
        const double* qp = &QNPH_DG[((size_t)jj * nfeds + L) * 2];
        double qnam = 0.5 * (qa[0] + qa[1]) + 0.5 * (qa[1] - qa[0]) * XEGP[i];
        double qnph = 0.5 * (qp[0] + qp[1]) + 0.5 * (qp[1] - qp[0]) * XEGP[i];
        qne = qne + qnam * rff * std::cos(argj - qnph);
        double qte = 0.0;
        qx_ex = -(ty * qne - ny * qte) / (nx * ty - ny * tx);
        qy_ex = -(-tx * qne + nx * qte) / (nx * ty - ny * tx);
      }
      for (int k = 0; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el, k) * phi_edge(k, i, led);
        qx_in = qx_in + qx(s, el, k) * phi_edge(k, i, led);
        qy_in = qy_in + qy(s, el, k) * phi_edge(k, i, led);
        hb_in = hb_in + hb(el, k) * phi_edge(k, i, led);
      }
      double f[3];
      llf_flux(*this, ze_in, ze_in, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_in, sfac_in, sfac_in, nx, ny, G, f);
      for (int k = 0; k < dofh; ++k) {
        double w = 2.0 * M_INV[k] / AREAS[el] * XLEN[ged] * phi_edge(k, i, led) * WEGP[i];
        rze(s, el, k) = rze(s, el, k) - w * f[0];
        rqx(s, el, k) = rqx(s, el, k) - w * f[1];
        rqy(s, el, k) = rqy(s, el, k) - w * f[2];
      }
    }
  }
}

// radiation_edge_hydro.F:20-263 (unpinned)
void Model::radiation_edges() {
  const int s = IRK - 1;
  for (int ged : NREDN) {
    int led = NEDSD[2 * ged], el = NEDEL[2 * ged];
    if (WDFLG[el] == 0) continue;
    double nx = COSNX[ged], ny = SINNX[ged], tx = -ny, ty = nx;
    for (int i = 0; i < NEGP; ++i) {
      double ze_in = ze(s, el, 0), qx_in = qx(s, el, 0), qy_in = qy(s, el, 0);
      double hb_in = BATHED[((size_t)el * 3 + led) * NEGP + i];
      double sfac_in = SFACED[((size_t)el * 3 + led) * NEGP + i];
      for (int k = 1; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el, k) * phi_edge(k, i, led);
        qx_in = qx_in + qx(s, el, k) * phi_edge(k, i, led);
        qy_in = qy_in + qy(s, el, k) * phi_edge(k, i, led);
      }
      double qn = qx_in * nx + qy_in * ny, qt = qx_in * tx + qy_in * ty;
      double qne = -qn + 2 * std::sqrt(G / (hb_in + ze_in)) * ze_in, qte = qt;
      double den = 1.0 / (nx * ty - ny * tx);
      double qx_ex = (ty * qne - ny * qte) * den, qy_ex = (-tx * qne + nx * qte) * den;
      double f[3];
      llf_flux(*this, ze_in, ze_in, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_in, sfac_in, sfac_in, nx, ny, G, f);
      for (int k = 0; k < dofh; ++k) {
        double w = 2.0 * M_INV[k] / AREAS[el] * XLEN[ged] * phi_edge(k, i, led) * WEGP[i];
        rze(s, el, k) = rze(s, el, k) - w * f[0];
        rqx(s, el, k) = rqx(s, el, k) - w * f[1];
        rqy(s, el, k) = rqy(s, el, k) - w * f[2];
      }
    }
  }
}

// ebarrier_edge_hydro.F:1-220
void Model::ebarrier_edges() {
  const int s = IRK - 1;
  for (size_t L = 0; L < NEBSEGN.size(); ++L) {
    int ged = NEBSEGN[L], led = NEDSD[2 * ged], el = NEDEL[2 * ged];
    if (WDFLG[el] == 0) continue;
    double nx = COSNX[ged], ny = SINNX[ged], tx = -ny, ty = nx;
    for (int i = 0; i < NEGP; ++i) {
      double ze_in = ze(s, el, 0), qx_in = qx(s, el, 0), qy_in = qy(s, el, 0);
      double hb_in = BATHED[((size_t)el * 3 + led) * NEGP + i];
      for (int k = 1; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el, k) * phi_edge(k, i, led);
        qx_in = qx_in + qx(s, el, k) * phi_edge(k, i, led);
        qy_in = qy_in + qy(s, el, k) * phi_edge(k, i, led);
      }
      double sfac_in = SFACED[((size_t)el * 3 + led) * NEGP + i];
      double above = ze_in - EBHT[L];
      double subsup = 2.0 * above / 3.0;
      double qne, qte;
      if (above < BARMIN) {
        qne = -(qx_in * nx + qy_in * ny);
        qte = qx_in * tx + qy_in * ty;
      } else {
        qne = RAMPDG * EBCFSP[L] * subsup * std::sqrt(subsup * G);
        qte = 0.0;
      }
      double qx_ex = (ty * qne - ny * qte) / (nx * ty - ny * tx);
      double qy_ex = (-tx * qne + nx * qte) / (nx * ty - ny * tx);
      double f[3];
      llf_flux(*this, ze_in, ze_in, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_in, sfac_in, sfac_in, nx, ny, G, f);
      for (int k = 0; k < dofh; ++k) {
        double w = 2.0 * M_INV[k] / AREAS[el] * XLEN[ged] * phi_edge(k, i, led) * WEGP[i];
        rze(s, el, k) = rze(s, el, k) - w * f[0];
        rqx(s, el, k) = rqx(s, el, k) - w * f[1];
        rqy(s, el, k) = rqy(s, el, k) - w * f[2];
      }
    }
  }
}

// ibarrier_edge_hydro.F:21-607.  The reference's stale exterior momentum on
// the "other" side of an overtopping weir (QX_EX/QY_EX are not recomputed)
// is kept, as is zero gravity on a dry receiving side.
void Model::ibarrier_edges() {
  const int s = IRK - 1;
  const int nseg = (int)NIBSEGN.size() / 2;
  for (int L = 0; L < nseg; ++L) {
    int gedb = NIBSEGN[2 * L], gedf = NIBSEGN[2 * L + 1];
    if (gedf < 0) continue;
    int ledb = NEDSD[2 * gedb], ledf = NEDSD[2 * gedf];
    int elb = NEDEL[2 * gedb], elf = NEDEL[2 * gedf];
    if (WDFLG[elb] == 0 && WDFLG[elf] == 0) continue;
    double nxb = COSNX[gedb], nyb = SINNX[gedb], nxf = COSNX[gedf], nyf = SINNX[gedf];
    double txb = -nyb, tyb = nxb, txf = -nyf, tyf = nxf;
    for (int i = 0; i < NEGP; ++i) {
      int gpb = i, gpf = NEGP - 1 - i;
      double zeb = ze(s, elb, 0), qxb = qx(s, elb, 0), qyb = qy(s, elb, 0);
      double hbb = BATHED[((size_t)elb * 3 + ledb) * NEGP + gpb];
      double zef = ze(s, elf, 0), qxf = qx(s, elf, 0), qyf = qy(s, elf, 0);
      double hbf = BATHED[((size_t)elf * 3 + ledf) * NEGP + gpf];
      for (int k = 1; k < dofh; ++k) {
        zeb = zeb + ze(s, elb, k) * phi_edge(k, gpb, ledb);
        qxb = qxb + qx(s, elb, k) * phi_edge(k, gpb, ledb);
        qyb = qyb + qy(s, elb, k) * phi_edge(k, gpb, ledb);
        zef = zef + ze(s, elf, k) * phi_edge(k, gpf, ledf);
        qxf = qxf + qx(s, elf, k) * phi_edge(k, gpf, ledf);
        qyf = qyf + qy(s, elf, k) * phi_edge(k, gpf, ledf);
      }
      double sfacb = SFACED[((size_t)elb * 3 + ledb) * NEGP + gpb];
      double sfacf = SFACED[((size_t)elf * 3 + ledf) * NEGP + gpf];
      double aboveb = 0.0, abovef = 0.0;
      if (WDFLG[elb] == 1) aboveb = zeb - IBHT[L];
      if (WDFLG[elf] == 1) abovef = zef - IBHT[L];
      double qbn = 0, qfn = 0, qbt = 0, qft = 0;
      int weir = 0;
      if ((abovef <= BARMIN) && (aboveb <= BARMIN)) {
        qbn = -(qxb * nxb + qyb * nyb); qfn = -(qxf * nxf + qyf * nyf);
        qbt = qxb * txb + qyb * tyb; qft = qxf * txf + qyf * tyf;
        weir = 0;
      } else if (std::fabs(abovef - aboveb) < BARMIN) {
        qbn = -(qxb * nxb + qyb * nyb); qfn = -(qxf * nxf + qyf * nyf);
        qbt = qxb * txb + qyb * tyb; qft = qxf * txf + qyf * tyf;
        weir = 0;
      } else {
        double subsupf = 2.0 * abovef / 3.0, subsupb = 2.0 * aboveb / 3.0;
        if (abovef > aboveb && abovef > BARMIN) {
          weir = 1;
          if (aboveb > subsupf) qfn = RAMPDG * IBCFSB[L] * aboveb * std::sqrt(2.0 * G * (abovef - aboveb));
          else qfn = RAMPDG * IBCFSP[L] * subsupf * std::sqrt(subsupf * G);
          qft = 0.0;
        } else if (aboveb > abovef && aboveb > BARMIN) {
          weir = -1;
          if (abovef > subsupb) qbn = RAMPDG * IBCFSB[L] * abovef * std::sqrt(2.0 * G * (aboveb - abovef));
          else qbn = RAMPDG * IBCFSP[L] * subsupb * std::sqrt(subsupb * G);
          qbt = 0.0;
        }
      }
      double fb[3] = {0, 0, 0}, ff[3] = {0, 0, 0};
      double qx_ex = 0.0, qy_ex = 0.0;
      bool done = false;
      if (weir <= 0) {
        qx_ex = (tyb * qbn - nyb * qbt) / (nxb * tyb - nyb * txb);
        qy_ex = (-txb * qbn + nxb * qbt) / (nxb * tyb - nyb * txb);
        llf_flux(*this, zeb, zeb, qxb, qx_ex, qyb, qy_ex, hbb, hbb, sfacb, sfacb, nxb, nyb, G, fb);
        if (weir < 0) {
          double g = (WDFLG[elf] == 0) ? 0.0 : G;
          llf_flux(*this, zef, zef, qxf, qx_ex, qyf, qy_ex, hbf, hbf, sfacf, sfacf, nxf, nyf, g, ff);
          done = true;
        }
      }
      if (!done && weir >= 0) {
        qx_ex = (tyf * qfn - nyf * qft) / (nxf * tyf - nyf * txf);
        qy_ex = (-txf * qfn + nxf * qft) / (nxf * tyf - nyf * txf);
        llf_flux(*this, zef, zef, qxf, qx_ex, qyf, qy_ex, hbf, hbf, sfacf, sfacf, nxf, nyf, G, ff);
        if (weir > 0) {
          double g = (WDFLG[elb] == 0) ? 0.0 : G;
          llf_flux(*this, zeb, zeb, qxb, qx_ex, qyb, qy_ex, hbb, hbb, sfacb, sfacb, nxb, nyb, g, fb);
        }
      }
      for (int k = 0; k < dofh; ++k) {
        double wb = 2.0 * M_INV[k] / AREAS[elb] * XLEN[gedb] * phi_edge(k, gpb, ledb) * WEGP[gpb];
        double wf = 2.0 * M_INV[k] / AREAS[elf] * XLEN[gedf] * phi_edge(k, gpf, ledf) * WEGP[gpf];
        rze(s, elb, k) = rze(s, elb, k) - wb * fb[0];
        rqx(s, elb, k) = rqx(s, elb, k) - wb * fb[1];
        rqy(s, elb, k) = rqy(s, elb, k) - wb * fb[2];
        rze(s, elf, k) = rze(s, elf, k) - wf * ff[0];
        rqx(s, elf, k) = rqx(s, elf, k) - wf * ff[1];
        rqy(s, elf, k) = rqy(s, elf, k) - wf * ff[2];
      }
    }
  }
}

// internal_edge_hydro.F:37-350
void Model::internal_edges() {
  const int s = IRK - 1;
  const int nieds = (int)NIEDN.size();
#pragma omp parallel for schedule(static)
  for (int L = 0; L < nieds; ++L) {
    int ged = NIEDN[L];
    int led_in = NEDSD[2 * ged], led_ex = NEDSD[2 * ged + 1];
    int el_in = NEDEL[2 * ged], el_ex = NEDEL[2 * ged + 1];
    if (WDFLG[el_in] == 0 && WDFLG[el_ex] == 0) continue;
    // [var][k]; every mode (the reference sums modes 1-3 only, which is its
    // p=2 defect; at p=1 the loops are the same)
    double rin[3][6] = {{0}}, rex[3][6] = {{0}};
    double nx = COSNX[ged], ny = SINNX[ged], tx = -ny, ty = nx;
    double edfac_in = XLEN[ged] / AREAS[el_in], edfac_ex = XLEN[ged] / AREAS[el_ex];
    for (int i = 0; i < NEGP; ++i) {
      int gp_in = i, gp_ex = NEGP - 1 - i;
      double ze_in = 0, qx_in = 0, qy_in = 0, ze_ex = 0, qx_ex = 0, qy_ex = 0;
      double hb_in = BATHED[((size_t)el_in * 3 + led_in) * NEGP + gp_in];
      double sfac_in = SFACED[((size_t)el_in * 3 + led_in) * NEGP + gp_in];
      double hb_ex = BATHED[((size_t)el_ex * 3 + led_ex) * NEGP + gp_ex];
      double sfac_ex = SFACED[((size_t)el_ex * 3 + led_ex) * NEGP + gp_ex];
      for (int k = 0; k < dofh; ++k) {
        ze_in = ze_in + ze(s, el_in, k) * phi_edge(k, gp_in, led_in);
        qx_in = qx_in + qx(s, el_in, k) * phi_edge(k, gp_in, led_in);
        qy_in = qy_in + qy(s, el_in, k) * phi_edge(k, gp_in, led_in);
        ze_ex = ze_ex + ze(s, el_ex, k) * phi_edge(k, gp_ex, led_ex);
        qx_ex = qx_ex + qx(s, el_ex, k) * phi_edge(k, gp_ex, led_ex);
        qy_ex = qy_ex + qy(s, el_ex, k) * phi_edge(k, gp_ex, led_ex);
      }
      double f[3];
      llf_flux(*this, ze_in, ze_ex, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_ex, sfac_in, sfac_ex, nx, ny, G, f);
      double f_hat_o = f[0], g_in = f[1], h_in = f[2], g_ex = f[1], h_ex = f[2];
      if (std::fabs(f[0]) > 1.0e-8) {
        if (WDFLG[el_in] == 0) {
          if (f[0] > 0.0) {
            double qne = qx_ex * nx + qy_ex * ny, qte = qx_ex * tx + qy_ex * ty;
            double qni = -qne, qti = qte;
            double den = nx * ty - ny * tx;
            double qxi = (ty * qni - ny * qti) / den, qyi = (-tx * qni + nx * qti) / den;
            llf_flux(*this, ze_ex, ze_ex, qxi, qx_ex, qyi, qy_ex, hb_ex, hb_ex, sfac_ex, sfac_ex, nx, ny, G, f);
            f_hat_o = f[0]; g_ex = f[1]; h_ex = f[2];
            g_in = 0.0; h_in = 0.0;
          } else {
            llf_flux(*this, ze_in, ze_ex, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_ex, sfac_in, sfac_ex, nx, ny, 0.0, f);
            g_in = f[1]; h_in = f[2];
          }
        } else if (WDFLG[el_ex] == 0) {
          if (f[0] < 0.0) {
            double qni = qx_in * nx + qy_in * ny, qti = qx_in * tx + qy_in * ty;
            double qne = -qni, qte = qti;
            double den = nx * ty - ny * tx;
            double qxe = (ty * qne - ny * qte) / den, qye = (-tx * qne + nx * qte) / den;
            llf_flux(*this, ze_in, ze_in, qx_in, qxe, qy_in, qye, hb_in, hb_in, sfac_in, sfac_in, nx, ny, G, f);
            f_hat_o = f[0]; g_in = f[1]; h_in = f[2];
            g_ex = 0.0; h_ex = 0.0;
          } else {
            llf_flux(*this, ze_in, ze_ex, qx_in, qx_ex, qy_in, qy_ex, hb_in, hb_ex, sfac_in, sfac_ex, nx, ny, 0.0, f);
            g_ex = f[1]; h_ex = f[2];
          }
        }
      }
      for (int k = 0; k < dofh; ++k) {
        double w_in = edfac_in * edgeq(k, gp_in, led_in);
        double w_ex = edfac_ex * edgeq(k, gp_ex, led_ex);
        rin[0][k] = rin[0][k] - w_in * f_hat_o;
        rin[1][k] = rin[1][k] - w_in * g_in;
        rin[2][k] = rin[2][k] - w_in * h_in;
        rex[0][k] = rex[0][k] + w_ex * f_hat_o;
        rex[1][k] = rex[1][k] + w_ex * g_ex;
        rex[2][k] = rex[2][k] + w_ex * h_ex;
      }
    }
    int ind_in = -1, ind_ex = -1;
    for (int k = 0; k < 3; ++k) {
      if (ELEM_EDGE[3 * el_ex + k] == ged) ind_ex = k;
      if (ELEM_EDGE[3 * el_in + k] == ged) ind_in = k;
    }
    for (int k = 0; k < dofh; ++k) {
      ze_edge[((size_t)el_ex * 3 + ind_ex) * dofh + k] = rex[0][k];
      qx_edge[((size_t)el_ex * 3 + ind_ex) * dofh + k] = rex[1][k];
      qy_edge[((size_t)el_ex * 3 + ind_ex) * dofh + k] = rex[2][k];
      ze_edge[((size_t)el_in * 3 + ind_in) * dofh + k] = rin[0][k];
      qx_edge[((size_t)el_in * 3 + ind_in) * dofh + k] = rin[1][k];
      qy_edge[((size_t)el_in * 3 + ind_in) * dofh + k] = rin[2][k];
    }
  }
}

// internal_edge_hydro.F:352-383
void Model::add_internal_flux() {
  const int s = IRK - 1;
#pragma omp parallel for schedule(static)
  for (int l = 0; l < NE; ++l) {
    for (int k = 0; k < dofh; ++k) {
      double zs = 0.0, xs = 0.0, ys = 0.0;
      for (int i = 0; i < 3; ++i) {
        zs = zs + ze_edge[((size_t)l * 3 + i) * dofh + k];
        xs = xs + qx_edge[((size_t)l * 3 + i) * dofh + k];
        ys = ys + qy_edge[((size_t)l * 3 + i) * dofh + k];
      }
      rze(s, l, k) = rze(s, l, k) + zs;
      rqx(s, l, k) = rqx(s, l, k) + xs;
      rqy(s, l, k) = rqy(s, l, k) + ys;
    }
    for (int i = 0; i < 3 * dofh; ++i) {
      ze_edge[(size_t)l * 3 * dofh + i] = 0.0; qx_edge[(size_t)l * 3 * dofh + i] = 0.0;
      qy_edge[(size_t)l * 3 * dofh + i] = 0.0;
    }
  }
}

// rhs_dg_hydro.F:18-473
void Model::rhs_dg_hydro() {
  const int s = IRK - 1;
  const double DTDPH = 1.0 / DTDP;
#pragma omp parallel for schedule(static)
  for (int L = 0; L < NE; ++L) {
    if (rainfall > 0) {
      double src = 7.0556e-6;
      if (rainfall > 1) src = 0.0;
      if (src > 0.0)
        for (int i = 0; i < NAGP; ++i)
          for (int k = 0; k < dofh; ++k)
            rze(s, L, k) = rze(s, L, k) + SRFAC[((size_t)L * dofh + k) * NAGP + i] * src;
    }
    if (WDFLG[L] == 0) continue;
    int n1 = NM[3 * L], n2 = NM[3 * L + 1], n3 = NM[3 * L + 2];
    double depth_c = hb(L, 0) + ze(s, L, 0);
    double fh_nl_c = 1.0 / (NLEQ * depth_c + LEQ);
    double dpsidx[3] = {0, 0, 0}, dpsidy[3] = {0, 0, 0};
    if (NWS != 0 || NTIP != 0)
      for (int a = 0; a < 3; ++a) {
        dpsidx[a] = DRPSI[a] * DRDX[L] + DSPSI[a] * DSDX[L];
        dpsidy[a] = DRPSI[a] * DRDY[L] + DSPSI[a] * DSDY[L];
      }
    for (int i = 0; i < NAGP; ++i) {
      double ze_in = ze(s, L, 0), qx_in = qx(s, L, 0), qy_in = qy(s, L, 0);
      double hb_in = BATH[(size_t)L * NAGP + i];
      double dhb_x = DBATHDX[(size_t)L * NAGP + i], dhb_y = DBATHDY[(size_t)L * NAGP + i];
      double sfq = SFAC_ELEM[(size_t)L * NAGP + i];
      double depth = 0.0;
      for (int k = 1; k < dofh; ++k) {
        ze_in = ze_in + ze(s, L, k) * PHI_AREA[k * NAGP + i];
        qx_in = qx_in + qx(s, L, k) * PHI_AREA[k * NAGP + i];
        qy_in = qy_in + qy(s, L, k) * PHI_AREA[k * NAGP + i];
        depth = ze_in + hb_in;
      }
      double F1_NL = NLEQ + LEQ * hb_in;
      double fx = qx_in * F1_NL * sfq;
      double fy = qy_in * F1_NL;
      double FU_NL = NLEQ * qx_in, FV_NL = NLEQ * qy_in;
      double FG_NL = NLEQG * ze_in * WDFLG[L];
      double FH_NL = 1.0 / (NLEQ * depth + LEQ);
      double u = qx_in * FH_NL, v = qy_in * FH_NL;
      double HUU = FU_NL * u, HVV = FV_NL * v, HUV = FU_NL * v;
      double GH2 = FG_NL * (0.5 * ze_in + hb_in) + FG_L * ze_in;
      double gx = (HUU + GH2) * sfq, gy = HUV;
      double hx = HUV * sfq, hy = HVV + GH2;
      if (LoadManningsN) {
        double nb = (ManningsN[n1] + ManningsN[n2] + ManningsN[n3]) / 3.;
        FRIC_EL[L] = G * (nb * nb) / pow_third_cr(depth);
        if (FRIC_EL[L] < CF) FRIC_EL[L] = CF;
      }
      double tau = FRIC_EL[L];
      if (IFLINBF == 0) {
        double umag = std::sqrt(u * u + v * v);
        tau = tau * umag * FH_NL;
        if (IFHYBF == 1) tau = tau * std::pow(1.0 + std::pow(HBREAK * fh_nl_c, FTHETA), FGAMMA / FTHETA);
        tau = std::min(tau, .9 * DTDPH);
      }
      double sx = -(tau * qx_in) + FG_NL * dhb_x * sfq + CORI_EL[L] * qy_in;
      double sy = -(tau * qy_in) + FG_NL * dhb_y - CORI_EL[L] * qx_in;
      if (NWS != 0) {
        double FW_NL = 1.0 / F1_NL;
        sx = sx + FW_NL * (WSX2[n1] * PSI1[i] + WSX2[n2] * PSI2[i] + WSX2[n3] * PSI3[i]) -
             G * sfq * depth * (PR2[n1] * dpsidx[0] + PR2[n2] * dpsidx[1] + PR2[n3] * dpsidx[2]);
        sy = sy + FW_NL * (WSY2[n1] * PSI1[i] + WSY2[n2] * PSI2[i] + WSY2[n3] * PSI3[i]) -
             G * depth * (PR2[n1] * dpsidy[0] + PR2[n2] * dpsidy[1] + PR2[n3] * dpsidy[2]);
      }
      size_t b0 = ((size_t)L * dofh) * NAGP + i;
      rqx(s, L, 0) = rqx(s, L, 0) + SRFAC[b0] * sx;
      rqy(s, L, 0) = rqy(s, L, 0) + SRFAC[b0] * sy;
      for (int k = 1; k < dofh; ++k) {
        size_t b = ((size_t)L * dofh + k) * NAGP + i;
        rze(s, L, k) = rze(s, L, k) + XFAC[b] * fx + YFAC[b] * fy;
        rqx(s, L, k) = rqx(s, L, k) + XFAC[b] * gx + YFAC[b] * gy + SRFAC[b] * sx;
        rqy(s, L, k) = rqy(s, L, k) + XFAC[b] * hx + YFAC[b] * hy + SRFAC[b] * sy;
      }
    }
  }
}

// DG_hydro_timestep.F:238-290
void Model::ssp_update() {
#pragma omp parallel for schedule(static)
  for (int j = 0; j < NE; ++j)
    for (int i = 1; i <= IRK; ++i) {
      double ark = atvd(IRK, i);
      double brk = btvd(IRK, i) * DTDP;
      for (int k = 0; k < dofh; ++k) {
        ze(IRK, j, k) = ze(IRK, j, k) + ark * ze(i - 1, j, k) + brk * rze(i - 1, j, k);
        qx(IRK, j, k) = qx(IRK, j, k) + ark * qx(i - 1, j, k) + brk * rqx(i - 1, j, k);
        qy(IRK, j, k) = qy(IRK, j, k) + ark * qy(i - 1, j, k) + brk * rqy(i - 1, j, k);
      }
    }
}

// slopelimiter.F:3259-3781 (SLOPELIMITER5)
void Model::slopelimiter5() {
  const int s = IRK;  // stage IRK+1
  std::vector<double> mn(6 * (size_t)NP);
#pragma omp parallel for schedule(static)
  for (int n = 0; n < NP; ++n) {
    double zmin = 99999., zmax = -99999., xmin = 99999., xmax = -99999., ymin = 99999., ymax = -99999.;
    for (int p = star_ptr[n]; p < star_ptr[n + 1]; ++p) {
      int e = star[p];
      double zt = ze(s, e, 0), xt = qx(s, e, 0), yt = qy(s, e, 0);
      zmin = std::min(zmin, zt); xmin = std::min(xmin, xt); ymin = std::min(ymin, yt);
      zmax = std::max(zmax, zt); xmax = std::max(xmax, xt); ymax = std::max(ymax, yt);
    }
    double* o = &mn[6 * (size_t)n];
    o[0] = zmin; o[1] = zmax; o[2] = xmin; o[3] = xmax; o[4] = ymin; o[5] = ymax;
  }
#pragma omp parallel for schedule(static)
  for (int I = 0; I < NE; ++I) {
    int nn[3] = {NM[3 * I], NM[3 * I + 1], NM[3 * I + 2]};
    for (int ivar = 0; ivar < 3; ++ivar) {
      double* c = (ivar == 0) ? &ze(s, I, 0) : (ivar == 1) ? &qx(s, I, 0) : &qy(s, I, 0);
      double zec[3] = {c[0], c[1], c[2]};
      double zmax1[3], zmin1[3];
      for (int a = 0; a < 3; ++a) {
        zmin1[a] = mn[6 * (size_t)nn[a] + 2 * ivar];
        zmax1[a] = mn[6 * (size_t)nn[a] + 2 * ivar + 1];
      }
      double vx[3] = {zec[0], zec[0], zec[0]};
      for (int kk = 1; kk < 3; ++kk)
        for (int a = 0; a < 3; ++a) vx[a] = vx[a] + phi_corner(kk, a) * zec[kk];
      for (int a = 0; a < 3; ++a) vx[a] = std::max(std::min(vx[a], zmax1[a]), zmin1[a]);
      for (int ll = 0; ll < 3; ++ll) {
        double sumloc = (vx[0] + vx[1] + vx[2]) / 3.0;
        double sumdif = (sumloc - zec[0]) * 3.0;
        double signdif = std::copysign(1.0, sumdif);
        double dif[3];
        for (int a = 0; a < 3; ++a) dif[a] = (vx[a] - zec[0]) * signdif;
        int kdp = (dif[0] > 0) + (dif[1] > 0) + (dif[2] > 0);
        for (int k = 0; k < 3; ++k) {
          double div = std::max(1.0, (double)kdp);
          double redfac;
          if (dif[k] > 0) { redfac = sumdif * signdif / div; kdp = kdp - 1; }
          else redfac = 0;
          double redmax = (signdif > 0) ? vx[k] - zmin1[k] : zmax1[k] - vx[k];
          redfac = std::min(redfac, redmax);
          sumdif = sumdif - redfac * signdif;
          vx[k] = vx[k] - redfac * signdif;
        }
      }
      c[1] = -(1.0 / 6.0 * (vx[0] + vx[1])) + 1.0 / 3.0 * vx[2];
      c[2] = -(.5 * vx[0]) + .5 * vx[1];
    }
  }
}

// wetdry.F:17-553 (p=1: pa=1)
void Model::wetdry() {
  const int s = IRK;
  const double ZERO = 1.0e-6, HUGEV = 1.0e6;
  for (int n = 0; n < NP; ++n) NODECODE[n] = 0;
  std::vector<char> setnode(NE, 0);
#pragma omp parallel for schedule(static)
  for (int J = 0; J < NE; ++J) {
    int ndry = 0, htmax_i = 0, htmin_i = 0;
    double htmin = HUGEV, htmax = ZERO;
    double ze_node[3], ht_node[3];
    for (int I = 0; I < 3; ++I) {
      ze_node[I] = ze(s, J, 0);
      for (int k = 1; k < dofh; ++k) ze_node[I] = ze_node[I] + phi_corner(k, I) * ze(s, J, k);
      ht_node[I] = DP_NODE[3 * J + I] + ze_node[I];
      if (ht_node[I] < htmin) { htmin_i = I; htmin = ht_node[I]; }
      if (ht_node[I] > htmax) { htmax_i = I; htmax = ht_node[I]; }
      if (ht_node[I] <= H0 + ZERO) ndry = ndry + 1;
    }
    (void)htmin_i;
    double dp_avg = C13 * (DP_NODE[3 * J] + DP_NODE[3 * J + 1] + DP_NODE[3 * J + 2]);
    double ze_hat[3] = {0, 0, 0};
    int element_check = 0;
    if (ndry == 0) {
      if (WDFLG[J] == 1) { element_check = 0; setnode[J] = 1; }
      else { for (int a = 0; a < 3; ++a) ze_hat[a] = ze_node[a]; element_check = 1; }
    } else if (ndry == 3) {
      double ht_avg = ze(s, J, 0) + dp_avg;
      for (int k = 0; k < dofh; ++k) ze(s, J, k) = 0.0;
      ze(s, J, 0) = ht_avg - dp_avg;
      if (ht_avg < ZERO) ze(s, J, 0) = ZERO - dp_avg;
      ze(s, J, 1) = -hb(J, 1);
      ze(s, J, 2) = -hb(J, 2);
      for (int k = 0; k < dofh; ++k) { qx(s, J, k) = 0.0; qy(s, J, k) = 0.0; }
      WDFLG[J] = 0;
      element_check = 0;
    } else {
      double ht_avg = ze(s, J, 0) + dp_avg;
      if (ht_avg <= H0 + ZERO) {
        for (int k = 0; k < dofh; ++k) ze(s, J, k) = 0.0;
        ze(s, J, 0) = ht_avg - dp_avg;
        if (ht_avg < ZERO) ze(s, J, 0) = ZERO - dp_avg;
        ze(s, J, 1) = -hb(J, 1);
        ze(s, J, 2) = -hb(J, 2);
        for (int a = 0; a < 3; ++a) ze_hat[a] = ze(s, J, 0);
        for (int k = 0; k < dofh; ++k) { qx(s, J, k) = 0.0; qy(s, J, k) = 0.0; }
      } else {
        int l2h[3] = {0, 1, 2};
        for (int k1 = 0; k1 < 3; ++k1)
          for (int k2 = k1; k2 < 3; ++k2)
            if (ht_node[l2h[k1]] > ht_node[l2h[k2]]) std::swap(l2h[k1], l2h[k2]);
        double dh[3];
        dh[l2h[0]] = std::max(H0, ht_node[l2h[0]]) - ht_node[l2h[0]];
        dh[l2h[1]] = std::max(H0, ht_node[l2h[1]] - 0.5 * dh[l2h[0]]) - ht_node[l2h[1]];
        dh[l2h[2]] = -dh[l2h[0]] - dh[l2h[1]];
        ndry = 0;
        double qxs = 0, qys = 0;
        htmax = 0;
        double ht_hat[3], qx_node[3], qy_node[3];
        for (int I = 0; I < 3; ++I) {
          ht_hat[I] = ht_node[I] + dh[I];
          qx_node[I] = qx(s, J, 0);
          qy_node[I] = qy(s, J, 0);
          if (ht_hat[I] > htmax) { htmax_i = I; htmax = ht_hat[I]; }
          for (int k = 1; k < dofh; ++k) {
            qx_node[I] = qx_node[I] + phi_corner(k, I) * qx(s, J, k);
            qy_node[I] = qy_node[I] + phi_corner(k, I) * qy(s, J, k);
          }
          if (ht_hat[I] <= H0 + 1.0e-10) { ndry = ndry + 1; qxs = qxs + qx_node[I]; qys = qys + qy_node[I]; }
        }
        if (ndry == 3) {
          for (int k = 0; k < dofh; ++k) { qx(s, J, k) = 0.0; qy(s, J, k) = 0.0; }
        } else {
          qxs = qxs / (3.0 - (double)ndry);
          qys = qys / (3.0 - (double)ndry);
          double qxh[3], qyh[3];
          for (int I = 0; I < 3; ++I) {
            if (ht_hat[I] <= H0 + 1.0e-10) { qxh[I] = 0.0; qyh[I] = 0.0; }
            else { qxh[I] = qx_node[I] + qxs; qyh[I] = qy_node[I] + qys; }
          }
          qx(s, J, 0) = C13 * (qxh[0] + qxh[1] + qxh[2]);
          qx(s, J, 1) = -(C16 * (qxh[0] + qxh[1])) + C13 * qxh[2];
          qx(s, J, 2) = -(0.5 * qxh[0]) + 0.5 * qxh[1];
          qy(s, J, 0) = C13 * (qyh[0] + qyh[1] + qyh[2]);
          qy(s, J, 1) = -(C16 * (qyh[0] + qyh[1])) + C13 * qyh[2];
          qy(s, J, 2) = -(0.5 * qyh[0]) + 0.5 * qyh[1];
        }
        for (int a = 0; a < 3; ++a) ze_hat[a] = ht_hat[a] - DP_NODE[3 * J + a];
        ze(s, J, 1) = -(C16 * (ze_hat[0] + ze_hat[1])) + C13 * ze_hat[2];
        ze(s, J, 2) = -(0.5 * ze_hat[0]) + 0.5 * ze_hat[1];
      }
      for (int k = 3; k < dofh; ++k) { ze(s, J, k) = 0.0; qx(s, J, k) = 0.0; qy(s, J, k) = 0.0; }
      element_check = 1;
    }
    if (element_check == 1) {
      if (ze_hat[htmax_i] > (-DPE_MIN[J] + H0)) {
        WDFLG[J] = 1;
        setnode[J] = 1;
      } else {
        for (int k = 0; k < dofh; ++k) { qx(s, J, k) = 0.0; qy(s, J, k) = 0.0; }
        WDFLG[J] = 0;
      }
    }
  }
  for (int J = 0; J < NE; ++J)
    if (setnode[J]) for (int a = 0; a < 3; ++a) NODECODE[NM[3 * J + a]] = 1;
}

// met_forcing.F:49-66: DO II = 1,NP: READ(22,*) NHG, WSX2(II), WSY2(II),
// PR2(II).  Each READ begins a new record and takes four values from it and,
// if it holds fewer, from the records that follow; what remains of its last
// record is skipped.  Blanks, tabs and commas separate values; a Fortran D
// exponent reads as E.
void Model::met_read_fort22() {
  WSX_BASE.resize(NP); WSY_BASE.resize(NP); PR_BASE.resize(NP);
  std::string line;
  for (int II = 0; II < NP; ++II) {
    double v[4];
    int got = 0;
    while (got < 4) {
      line.clear();
      int c;
      bool any = false;
      while ((c = std::fgetc(F22)) != EOF && c != '\n') { any = true; line.push_back((char)c); }
      if (!any && c == EOF) throw Err(F22_path + ": end of file (NWS = 1 reads NP records per stage)");
      for (char& ch : line) {
        if (ch == 'D' || ch == 'd') ch = 'E';
        if (ch == ',' || ch == '\t' || ch == '\r') ch = ' ';
      }
      std::istringstream is(line);
      std::string tok;
      while (got < 4 && (is >> tok)) {
        char* e = nullptr;
        v[got] = std::strtod(tok.c_str(), &e);
        if (e == tok.c_str() || *e) throw Err(F22_path + ": not a number: " + tok);
        ++got;
      }
    }
    WSX_BASE[II] = v[1];
    WSY_BASE[II] = v[2];
    PR_BASE[II] = v[3];
  }
}

// DG_hydro_timestep.F:24-744
void Model::step(int IT) {
  double ITDT = IT * DTDP;
  double TIME_A = ITDT + STATIM * 86400.0;
  for (IRK = 1; IRK <= NRK; ++IRK) {
    TIMEDG = TIME_A - DTDP + DTVD[IRK - 1] * DTDP;
    RAMPDG = 1.0;
    if (NRAMP == 1 || NRAMP == 2)
      RAMPDG = std::tanh((2.0 * ((IT - 1) + DTVD[IRK - 1]) * DTDP / 86400.0) / DRAMP);
    if (NRAMP == 3) throw Err("NRAMP = 3 not supported");
    if (NWS == 1 && F22) met_read_fort22();
    if (NWS == 1)
      for (int n = 0; n < NP; ++n) {
        WSX2[n] = RAMPDG * (WSX_BASE.empty() ? 0.0 : WSX_BASE[n]);
        WSY2[n] = RAMPDG * (WSY_BASE.empty() ? 0.0 : WSY_BASE[n]);
        PR2[n] = RAMPDG * (PR_BASE.empty() ? 0.0 : PR_BASE[n]);
      }
    if (!NEEDN.empty()) ocean_edges();
    if (!NLEDN.empty()) land_edges();
    if (!NFEDN.empty()) flow_edges();
    if (!NREDN.empty()) radiation_edges();
    if (!NIBSEGN.empty()) ibarrier_edges();
    if (!NEBSEGN.empty()) ebarrier_edges();
    internal_edges();
    add_internal_flux();
    rhs_dg_hydro();
    ssp_update();
    if (slopeflag != 0) slopelimiter5();
    if (NOLIFA >= 2) wetdry();
  }
  IRK = NRK;
  for (int j = 0; j < NE; ++j)
    for (int k = 0; k < dofh; ++k) {
      ze(0, j, k) = ze(NRK, j, k); qx(0, j, k) = qx(NRK, j, k); qy(0, j, k) = qy(NRK, j, k);
    }
  std::fill(ZE.begin() + (size_t)NE * dofh, ZE.end(), 0.0);
  std::fill(QX.begin() + (size_t)NE * dofh, QX.end(), 0.0);
  std::fill(QY.begin() + (size_t)NE * dofh, QY.end(), 0.0);
  std::fill(RHS_ZE.begin(), RHS_ZE.end(), 0.0);
  std::fill(RHS_QX.begin(), RHS_QX.end(), 0.0);
  std::fill(RHS_QY.begin(), RHS_QY.end(), 0.0);
}

// write_results.F:14-170 (modal2nodal), star in element order
void Model::modal2nodal(double* eta2, double* uu2, double* vv2) const {
  for (int I = 0; I < NP; ++I) {
    double area_sum = 0;
    for (int p = star_ptr[I]; p < star_ptr[I + 1]; ++p) {
      int e = star[p];
      if (WDFLG[e] == 0) continue;
      area_sum = area_sum + 0.5 * AREAS[e];
    }
    double et = 0.0, uu = 0.0, vv = 0.0;
    for (int p = star_ptr[I]; p < star_ptr[I + 1]; ++p) {
      int e = star[p];
      if (WDFLG[e] == 0) continue;
      int K = 0;
      while (K < 3 && NM[3 * e + K] != I) ++K;
      double zd = ZE[(size_t)e * dofh], xd = QX[(size_t)e * dofh], yd = QY[(size_t)e * dofh];
      double hd = HB[(size_t)e * dofh];
      for (int kk = 1; kk < dofh; ++kk) {
        double pc = PHI_CORNER[K * dofh + kk];
        zd = zd + pc * ZE[(size_t)e * dofh + kk];
        xd = xd + pc * QX[(size_t)e * dofh + kk];
        yd = yd + pc * QY[(size_t)e * dofh + kk];
        hd = hd + pc * HB[(size_t)e * dofh + kk];
      }
      double area = 0.50 * AREAS[e] / area_sum;
      double depth = zd + hd;
      double fh = 1.0 / (NLEQ * depth + LEQ);
      et = et + area * zd;
      uu = uu + area * xd * fh;
      vv = vv + area * yd * fh;
    }
    if (eta2) eta2[I] = et;
    if (uu2) uu2[I] = uu;
    if (vv2) vv2[I] = vv;
  }
}

static void copy_err(const std::string& s, char* err, int errlen) {
  if (err && errlen > 0) {
    std::strncpy(err, s.c_str(), (size_t)errlen - 1);
    err[errlen - 1] = 0;
  }
}

}  // namespace orc

struct orc_model {
  orc::Model m;
};

extern "C" {

void orc_pow_third(const double* xs, long n, double* out) {
  for (long i = 0; i < n; ++i) out[i] = orc::pow_third_cr(xs[i]);
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

orc_model* orc_open(const char* dir, char* err, int errlen) {
  orc_model* h = new orc_model();
  try {
    h->m.read_fort_dg(dir);
    h->m.read_input(dir);
    h->m.prep_dg();
    if (h->m.NWS == 1) {
      h->m.F22_path = std::string(dir) + "/fort.22";
      h->m.F22 = std::fopen(h->m.F22_path.c_str(), "rb");  // optional: orc_set_met gives the fields otherwise
    }
  } catch (std::exception& e) {
    orc::copy_err(e.what(), err, errlen);
    delete h;
    return nullptr;
  }
  return h;
}

void orc_close(orc_model* m) { delete m; }

int orc_info_int(const orc_model* h, const char* key) {
  const orc::Model& m = h->m;
  std::string k(key);
  if (k == "ne") return m.NE;
  if (k == "np") return m.NP;
  if (k == "dofh") return m.dofh;
  if (k == "nrk") return m.NRK;
  if (k == "nt") return m.NT;
  if (k == "nedges") return m.NEDGES;
  if (k == "nieds") return (int)m.NIEDN.size();
  if (k == "nleds") return (int)m.NLEDN.size();
  if (k == "needs") return (int)m.NEEDN.size();
  if (k == "nfeds") return (int)m.NFEDN.size();
  if (k == "nreds") return (int)m.NREDN.size();
  if (k == "nebseg") return (int)m.NEBSEGN.size();
  if (k == "nibseg") return (int)m.NIBSEGN.size() / 2;
  if (k == "nspoolge") return m.NSPOOLGE;
  if (k == "ntcysge") return m.NTCYSGE;
  if (k == "ntcyfge") return m.NTCYFGE;
  if (k == "nolifa") return m.NOLIFA;
  if (k == "slopeflag") return m.slopeflag;
  if (k == "ics") return m.ICS;
  if (k == "nws") return m.NWS;
  if (k == "rainfall") return m.rainfall;
  if (k == "ph") return m.ph;
  return -1;
}

double orc_info_real(const orc_model* h, const char* key) {
  const orc::Model& m = h->m;
  std::string k(key);
  if (k == "dtdp") return m.DTDP;
  if (k == "g") return m.G;
  if (k == "h0") return m.H0;
  if (k == "statim") return m.STATIM;
  return 0.0;
}

int orc_step(orc_model* h, int it) {
  try { h->m.step(it); } catch (std::exception&) { return 1; }
  return 0;
}

int orc_run(orc_model* h, int it0, int it1) {
  for (int it = it0; it <= it1; ++it)
    if (orc_step(h, it)) return 1;
  return 0;
}

void orc_get_state(const orc_model* h, double* ze, double* qx, double* qy, int* wdflg) {
  const orc::Model& m = h->m;
  size_t n = (size_t)m.NE * m.dofh;
  if (ze) std::memcpy(ze, m.ZE.data(), n * sizeof(double));
  if (qx) std::memcpy(qx, m.QX.data(), n * sizeof(double));
  if (qy) std::memcpy(qy, m.QY.data(), n * sizeof(double));
  if (wdflg) std::memcpy(wdflg, m.WDFLG.data(), (size_t)m.NE * sizeof(int));
}

void orc_set_state(orc_model* h, const double* ze, const double* qx, const double* qy, const int* wdflg) {
  orc::Model& m = h->m;
  size_t n = (size_t)m.NE * m.dofh;
  if (ze) std::memcpy(m.ZE.data(), ze, n * sizeof(double));
  if (qx) std::memcpy(m.QX.data(), qx, n * sizeof(double));
  if (qy) std::memcpy(m.QY.data(), qy, n * sizeof(double));
  if (wdflg) std::memcpy(m.WDFLG.data(), wdflg, (size_t)m.NE * sizeof(int));
}

void orc_get_hb(const orc_model* h, double* hb) {
  std::memcpy(hb, h->m.HB.data(), h->m.HB.size() * sizeof(double));
}

void orc_get_nodecode(const orc_model* h, int* nc) {
  std::memcpy(nc, h->m.NODECODE.data(), h->m.NODECODE.size() * sizeof(int));
}

void orc_modal2nodal(const orc_model* h, double* eta2, double* uu2, double* vv2) {
  h->m.modal2nodal(eta2, uu2, vv2);
}

void orc_set_met(orc_model* h, const double* wsx, const double* wsy, const double* pr) {
  orc::Model& m = h->m;
  if (m.F22) { std::fclose(m.F22); m.F22 = nullptr; }  // the given fields replace the deck's fort.22
  m.WSX_BASE.assign(wsx, wsx + m.NP);
  m.WSY_BASE.assign(wsy, wsy + m.NP);
  m.PR_BASE.assign(pr, pr + m.NP);
}

int orc_get_int_table(const orc_model* h, const char* which, int* out, int cap) {
  const orc::Model& m = h->m;
  std::string w(which);
  std::vector<int> v;
  auto plus1 = [](const std::vector<int>& a) {
    std::vector<int> r(a.size());
    for (size_t i = 0; i < a.size(); ++i) r[i] = a[i] + 1;  // -1 -> 0 as in Fortran
    return r;
  };
  if (w == "NEDNO") v = plus1(m.NEDNO);
  else if (w == "NEDEL") v = plus1(m.NEDEL);
  else if (w == "NELED") v = plus1(m.NELED);
  else if (w == "NEDSD") v = plus1(m.NEDSD);
  else if (w == "NIEDN") v = plus1(m.NIEDN);
  else if (w == "NLEDN") v = plus1(m.NLEDN);
  else if (w == "NEEDN") v = plus1(m.NEEDN);
  else if (w == "NFEDN") v = plus1(m.NFEDN);
  else if (w == "NREDN") v = plus1(m.NREDN);
  else if (w == "NEBSEGN") v = plus1(m.NEBSEGN);
  else if (w == "NIBSEGN") v = plus1(m.NIBSEGN);
  else if (w == "ELEM_EDGE") v = plus1(m.ELEM_EDGE);
  else if (w == "WDFLG") v = m.WDFLG;
  else return -1;
  int n = (int)v.size();
  if (out) std::memcpy(out, v.data(), (size_t)std::min(n, cap) * sizeof(int));
  return n;
}

int orc_get_real_table(const orc_model* h, const char* which, double* out, int cap) {
  const orc::Model& m = h->m;
  std::string w(which);
  const std::vector<double>* v = nullptr;
  if (w == "XLEN") v = &m.XLEN;
  else if (w == "COSNX") v = &m.COSNX;
  else if (w == "SINNX") v = &m.SINNX;
  else if (w == "AREAS") v = &m.AREAS;
  else if (w == "DP") v = &m.DP;
  else if (w == "X") v = &m.X;
  else if (w == "Y") v = &m.Y;
  else if (w == "HB") v = &m.HB;
  // basis and area rule (p-generic): PHI_AREA[k*NAGP + i], the reference
  // triangle's area points and weights (weights sum to 2), M_INV per mode
  else if (w == "PHI_AREA") v = &m.PHI_AREA;
  else if (w == "XAGP") v = &m.XAGP;
  else if (w == "YAGP") v = &m.YAGP;
  else if (w == "WAGP") v = &m.WAGP;
  else if (w == "M_INV") v = &m.M_INV;
  else return -1;
  int n = (int)v->size();
  if (out) std::memcpy(out, v->data(), (size_t)std::min(n, cap) * sizeof(double));
  return n;
}

// dgswem.F:341-373 time loop + write_results.F:445-500 (fort.63 block)
int orc_run_case(const char* dir, const char* out_path, char* err, int errlen) {
  orc_model* h = orc_open(dir, err, errlen);
  if (!h) return 1;
  orc::Model& m = h->m;
  FILE* f = std::fopen(out_path, "w");
  if (!f) { orc::copy_err("cannot write output", err, errlen); orc_close(h); return 1; }
  int nsets = (m.NSPOOLGE > 0) ? (m.NTCYFGE - m.NTCYSGE) / m.NSPOOLGE : 0;
  std::fprintf(f, "%-32s  %-24s  %-24s\n", m.RUNDES.substr(0, 32).c_str(),
               m.RUNID.substr(0, 24).c_str(), m.AGRID.substr(0, 24).c_str());
  std::fprintf(f, " %10d %10d %15.7E %5d %5d\n", nsets, m.NP, m.DTDP * m.NSPOOLGE, m.NSPOOLGE, 1);
  std::vector<double> eta(m.NP);
  int nscouge = 0;
  for (int it = 1; it <= m.NT; ++it) {
    if (orc_step(h, it)) { orc::copy_err("step failed", err, errlen); std::fclose(f); orc_close(h); return 1; }
    if (m.NOUTGE != 0 && it > m.NTCYSGE && it <= m.NTCYFGE) {
      ++nscouge;
      if (nscouge == m.NSPOOLGE) {
        m.modal2nodal(eta.data(), nullptr, nullptr);
        double time_a = it * m.DTDP + m.STATIM * 86400.0;
        std::fprintf(f, "  %20.10E     %10d\n", time_a, it);
        for (int i = 0; i < m.NP; ++i) {
          double v = eta[i];
          if (std::fabs(v) <= 1e-30) v = 0.0;
          if (m.NOLIFA == 2 && m.NODECODE[i] == 0) v = -99999.;
          std::fprintf(f, "  %8d  %16.8E\n", i + 1, v);
        }
        nscouge = 0;
      }
    }
  }
  std::fclose(f);
  orc_close(h);
  return 0;
}

}  // extern "C"
