// hydro.cu -- libdgswem_cuda: device layout, launch sequence and C-ABI entry
// points of the B200 DG hydro time step (declared in include/dgswem_cuda.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "abi_util.h"
#include "dgswem_cuda.h"
#include "hydro_device.cuh"
#include "partition.h"

namespace dgswem {

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

#define DG_CUDA(call)                                                                     \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      throw Failure(DGSWEM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// p=1 basis at the quadrature, edge and corner points (orthogonal_basis_v1.F
// recurrences evaluated for D=1, with the |value| < 1e-15 -> 0 rule)
static void p1_basis(double x, double y, double phi[3], double dr[3], double ds[3]) {
  double v[3] = {1.0, (1.0 + 3.0 * y) / 2.0, (1.0 + 2.0 * x + y) / 2.0};
  double a[3] = {0.0, 0.0, 1.0}, b[3] = {0.0, 3.0 / 2.0, 1.0 / 2.0};
  for (int k = 0; k < 3; ++k) {
    phi[k] = std::fabs(v[k]) < 1.0e-15 ? 0.0 : v[k];
    if (dr) dr[k] = a[k];
    if (ds) ds[k] = b[k];
  }
}

static BasisP1 make_basis_p1() {
  BasisP1 B{};
  // 3-point area rule (quadrature_v1.F:255-260, 802-840)
  const double A = 0.1666666666666666666666666666666666, W = 0.3333333333333333333333333333333333;
  const double C = 1.0 - (A + A);
  const double bary[3][3] = {{A, A, C}, {A, C, A}, {C, A, A}};
  for (int i = 0; i < 3; ++i) {
    const double x = -1.0 * bary[i][0] + 1.0 * bary[i][1] + -1.0 * bary[i][2];
    const double y = -1.0 * bary[i][0] + -1.0 * bary[i][1] + 1.0 * bary[i][2];
    double phi[3], dr[3], ds[3];
    p1_basis(x, y, phi, dr, ds);
    for (int k = 0; k < 3; ++k) {
      B.phi_area[k][i] = phi[k];
      B.drphi[k][i] = dr[k];
      B.dsphi[k][i] = ds[k];
    }
    B.wagp[i] = 2.0 * W;
    B.psi[0][i] = -1.0 / 2.0 * (x + y);
    B.psi[1][i] = 1.0 / 2.0 * (x + 1.0);
    B.psi[2][i] = 1.0 / 2.0 * (y + 1.0);
  }
  // 3-point Gauss-Lobatto edge rule (quad_rules_general.F)
  B.xegp[0] = -1.0; B.xegp[1] = 0.0; B.xegp[2] = 1.0;
  B.wegp[0] = 2.0 / ((1.0 + 1.0) * (1.0 + 2.0));
  B.wegp[2] = B.wegp[0];
  {
    const double p2 = ((2.0 * 1.0 + 1.0) * 0.0 * 0.0 - 1.0 * 1.0) / (1.0 + 1.0);
    B.wegp[1] = 2.0 / ((1.0 + 1.0) * (1.0 + 2.0) * p2 * p2);
  }
  // M_INV (prep_DG.F:712-721): (I,JJ) = (0,0),(0,1),(1,0)
  B.m_inv[0] = (2.0 * 0 + 1.0) * (2.0 * 0 + 2.0 * 0 + 2.0) / 4.0;
  B.m_inv[1] = (2.0 * 0 + 1.0) * (2.0 * 1 + 2.0 * 0 + 2.0) / 4.0;
  B.m_inv[2] = (2.0 * 1 + 1.0) * (2.0 * 0 + 2.0 * 1 + 2.0) / 4.0;
  // edge points: edge 1 (-x, x), edge 2 (-1, -x), edge 3 (x, -1)
  for (int l = 0; l < 3; ++l)
    for (int j = 0; j < 3; ++j) {
      const double t = B.xegp[j];
      const double px = l == 0 ? -t : (l == 1 ? -1.0 : t);
      const double py = l == 0 ? t : (l == 1 ? -t : -1.0);
      double phi[3];
      p1_basis(px, py, phi, nullptr, nullptr);
      for (int k = 0; k < 3; ++k) {
        B.phi_edge[l][j][k] = phi[k];
        B.edgeq[l][j][k] = 2.0 * B.m_inv[k] * phi[k] * B.wegp[j];
      }
    }
  const double vx[3] = {-1.0, 1.0, -1.0}, vy[3] = {-1.0, -1.0, 1.0};
  for (int v = 0; v < 3; ++v) p1_basis(vx[v], vy[v], B.phi_corner[v], nullptr, nullptr);
  // products the kernels form left to right, M_INV * WAGP (* PHI_AREA)
  for (int k = 0; k < 3; ++k)
    for (int i = 0; i < 3; ++i) {
      B.mw[k][i] = B.m_inv[k] * B.wagp[i];
      B.srfac[k][i] = B.m_inv[k] * B.wagp[i] * B.phi_area[k][i];
    }
  return B;
}

// Orthogonal basis of degree <= 2 on the reference triangle and its r/s
// derivatives at (X, Y), in the hierarchical order (P, Q-P), Q = 0..D,
// P = 0..Q (orthogonal_basis_v1.F:50-244: the Jacobi-type recurrences in P
// and Q, values below 1e-15 set to 0).
static void ortho_basis_p2(double X, double Y, double* b, double* d1, double* d2) {
  constexpr int D = 2;
  double PHI[D + 1][D + 1] = {}, DP1[D + 1][D + 1] = {}, DP2[D + 1][D + 1] = {};
  PHI[0][0] = 1.0;
  PHI[1][0] = (1.0 + 2.0 * X + Y) / 2.0;
  DP1[1][0] = 1.0;
  DP2[1][0] = 1.0 / 2.0;
  for (int P = 1; P <= D - 1; ++P) {
    const double w = (1.0 - Y) / 2.0;
    const double a = (2.0 * P + 1.0) / (P + 1.0), c = P / (P + 1.0);
    PHI[P + 1][0] = a * PHI[1][0] * PHI[P][0] - c * (w * w) * PHI[P - 1][0];
    DP1[P + 1][0] = a * (DP1[1][0] * PHI[P][0] + PHI[1][0] * DP1[P][0]) - c * (w * w) * DP1[P - 1][0];
    DP2[P + 1][0] = a * (DP2[1][0] * PHI[P][0] + PHI[1][0] * DP2[P][0]) -
                    c * ((Y - 1) / 2 * PHI[P - 1][0] + (w * w) * DP2[P - 1][0]);
  }
  for (int P = 0; P <= D - 1; ++P) {
    const double f = (1.0 + 2.0 * P + (3.0 + 2.0 * P) * Y) / 2.0;
    PHI[P][1] = PHI[P][0] * f;
    DP1[P][1] = DP1[P][0] * f;
    DP2[P][1] = DP2[P][0] * f + PHI[P][0] * (3.0 + 2.0 * P) / 2.0;
  }
  for (int Q = 1; Q <= D - 1; ++Q)
    for (int P = 0; P <= D - Q - 1; ++P) {
      const double AQ = (2.0 * Q + 2.0 + 2.0 * P) * (2.0 * Q + 3.0 + 2.0 * P) / (2.0 * Q + 2.0) / (Q + 2.0 + 2.0 * P);
      const double t = 2.0 * P + 1.0;
      const double BQ = (t * t) * (2.0 * Q + 2.0 + 2.0 * P) / (2.0 * Q + 2.0) / (2.0 * Q + 2.0 * P + 1.0) /
                        (Q + 2.0 + 2.0 * P);
      const double CQ = (Q + 2.0 * P + 1.0) * Q * (2.0 * Q + 3.0 + 2.0 * P) / (Q + 1.0) / (Q + 2.0 + 2.0 * P) /
                        (2.0 * Q + 2.0 * P + 1.0);
      PHI[P][Q + 1] = (AQ * Y + BQ) * PHI[P][Q] - CQ * PHI[P][Q - 1];
      DP1[P][Q + 1] = (AQ * Y + BQ) * DP1[P][Q] - CQ * DP1[P][Q - 1];
      DP2[P][Q + 1] = (AQ * Y + BQ) * DP2[P][Q] + AQ * PHI[P][Q] - CQ * DP2[P][Q - 1];
    }
  int k = 0;
  for (int Q = 0; Q <= D; ++Q)
    for (int P = 0; P <= Q; ++P, ++k) {
      const double v0 = PHI[P][Q - P], v1 = DP1[P][Q - P], v2 = DP2[P][Q - P];
      b[k] = std::fabs(v0) < 1.0e-15 ? 0.0 : v0;
      if (d1) d1[k] = std::fabs(v1) < 1.0e-15 ? 0.0 : v1;
      if (d2) d2[k] = std::fabs(v2) < 1.0e-15 ? 0.0 : v2;
    }
}

// p=2 tables: the six-point area rule of degree 4 (quadrature_v1.F:245-262,
// 802-840: two orbits of barycentric points on the reference triangle
// (-1,-1), (1,-1), (-1,1), weights doubled to its area 2), the four-point
// Gauss-Lobatto edge rule (quad_rules_general.F: +-1, +-sqrt(1/5), weights
// from the Legendre polynomial of degree 3), M_INV, PHI_EDGE and EDGEQ as
// prep_DG.F:648-870 builds them.
static BasisP2 make_basis_p2() {
  BasisP2 B{};
  const double V1[2] = {-1.0, -1.0}, V2[2] = {1.0, -1.0}, V3[2] = {-1.0, 1.0};
  const double Av[2] = {0.4459484909159648863183292538830519, 0.0915762135097707434595714634022015};
  const double Wv[2] = {0.2233815896780114656950070084331228, 0.1099517436553218676383263249002105};
  double xa[kP2Agp], ya[kP2Agp];
  int n = 0;
  for (int o = 0; o < 2; ++o) {
    const double a = Av[o], b = Av[o], c = 1.0 - (a + b);
    const double tri[3][3] = {{a, b, c}, {b, c, a}, {c, a, b}};
    for (int r = 0; r < 3; ++r, ++n) {
      xa[n] = V1[0] * tri[r][0] + V2[0] * tri[r][1] + V3[0] * tri[r][2];
      ya[n] = V1[1] * tri[r][0] + V2[1] * tri[r][1] + V3[1] * tri[r][2];
      B.wagp[n] = 2.0 * Wv[o];
    }
  }
  for (int i = 0; i < kP2Agp; ++i) {
    double phi[kP2Modes], dr[kP2Modes], ds[kP2Modes];
    ortho_basis_p2(xa[i], ya[i], phi, dr, ds);
    for (int k = 0; k < kP2Modes; ++k) {
      B.phi_area[k][i] = phi[k];
      B.drphi[k][i] = dr[k];
      B.dsphi[k][i] = ds[k];
    }
    B.psi[0][i] = -1.0 / 2.0 * (xa[i] + ya[i]);
    B.psi[1][i] = 1.0 / 2.0 * (xa[i] + 1.0);
    B.psi[2][i] = 1.0 / 2.0 * (ya[i] + 1.0);
  }
  {
    const double sq = std::sqrt(1.0 / 5.0), nrl = 2.0;
    B.xegp[0] = -1.0; B.xegp[1] = -sq; B.xegp[2] = sq; B.xegp[3] = 1.0;
    B.wegp[0] = 2.0 / ((nrl + 1.0) * (nrl + 2.0));
    B.wegp[3] = B.wegp[0];
    for (int m = 1; m <= 2; ++m) {
      const double x = B.xegp[m];
      double pm1 = 1.0, pc = x;
      for (int q = 1; q <= 2; ++q) {
        const double pn = ((2.0 * q + 1.0) * x * pc - q * pm1) / (q + 1.0);
        pm1 = pc;
        pc = pn;
      }
      B.wegp[m] = 2.0 / ((nrl + 1.0) * (nrl + 2.0) * pc * pc);
    }
  }
  {
    int k = 0;
    for (int J = 0; J <= 2; ++J)
      for (int I = 0; I <= J; ++I, ++k) {
        const int JJ = J - I;
        B.m_inv[k] = (2.0 * I + 1.0) * (2.0 * JJ + 2.0 * I + 2.0) / 4.0;
      }
  }
  for (int l = 0; l < 3; ++l)
    for (int q = 0; q < kP2Egp; ++q) {
      const double t = B.xegp[q];
      const double px = l == 0 ? -t : (l == 1 ? -1.0 : t);
      const double py = l == 0 ? t : (l == 1 ? -t : -1.0);
      double phi[kP2Modes];
      ortho_basis_p2(px, py, phi, nullptr, nullptr);
      for (int k = 0; k < kP2Modes; ++k) {
        B.phi_edge[l][q][k] = phi[k];
        B.edgeq[l][q][k] = 2.0 * B.m_inv[k] * phi[k] * B.wegp[q];
      }
    }
  const double vx[3] = {-1.0, 1.0, -1.0}, vy[3] = {-1.0, -1.0, 1.0};
  for (int v = 0; v < 3; ++v) ortho_basis_p2(vx[v], vy[v], B.phi_corner[v], nullptr, nullptr);
  for (int k = 0; k < kP2Modes; ++k)
    for (int i = 0; i < kP2Agp; ++i) {
      B.mw[k][i] = B.m_inv[k] * B.wagp[i];
      B.srfac[k][i] = B.m_inv[k] * B.wagp[i] * B.phi_area[k][i];
    }
  return B;
}

// Owning device allocation; movable, not copyable (a copy would free the
// buffer twice).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) DG_CUDA(cudaMalloc(&p, count * sizeof(T)));
  }
  void ensure(size_t count) {  // grow only
    if (count > n) alloc(count);
  }
  void upload(const std::vector<T>& v) {
    alloc(v.size());
    if (n) DG_CUDA(cudaMemcpy(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
};

// Launchers of one compilation variant (kernels_fast.cu / kernels_strict.cu /
// kernels_mixed.cu) and the byte size of its stage kernel's arithmetic type.
struct Variant {
  unsigned real_bytes;
  void (*set_basis)(const BasisP1&);
  void (*stage)(const StageArgs&, bool, int, unsigned, size_t, cudaStream_t);
  void (*ibarrier)(const StageArgs&, bool, cudaStream_t);
  void (*node_minmax)(const LimitArgs&, unsigned, cudaStream_t);
  void (*limit_wetdry)(const LimitArgs&, int, cudaStream_t);
  void (*modal2nodal)(const MeshView&, const double*, const int*, double, double, double*, double*,
                      double*, int*, unsigned, cudaStream_t);
  void (*f2s)(const double*, double*, int, int, const int*, unsigned, cudaStream_t);
  void (*s2f)(const double*, double*, int, int, const int*, unsigned, cudaStream_t);
  void (*gather_int)(const int*, int*, const int*, int, unsigned, cudaStream_t);
  void (*halo)(bool, double*, int*, int, const int*, int, int, double*, cudaStream_t);
};

static const Variant kFast = {8, fast::set_basis, fast::launch_stage, fast::launch_ibarrier, fast::launch_node_minmax,
                              fast::launch_limit_wetdry, fast::launch_modal2nodal,
                              fast::launch_fortran_to_soa, fast::launch_soa_to_fortran, fast::launch_gather_int,
                              fast::launch_halo};
static const Variant kStrict = {8, strict::set_basis, strict::launch_stage, strict::launch_ibarrier, strict::launch_node_minmax,
                                strict::launch_limit_wetdry, strict::launch_modal2nodal,
                                strict::launch_fortran_to_soa, strict::launch_soa_to_fortran,
                                strict::launch_gather_int, strict::launch_halo};
static const Variant kMixed = {4, mixed::set_basis, mixed::launch_stage, mixed::launch_ibarrier, mixed::launch_node_minmax,
                               mixed::launch_limit_wetdry, mixed::launch_modal2nodal,
                               mixed::launch_fortran_to_soa, mixed::launch_soa_to_fortran,
                               mixed::launch_gather_int, mixed::launch_halo};

// Launchers of the p=2 stage (kernels_p2_fast.cu / kernels_p2_strict.cu /
// kernels_p2_mixed.cu)
struct P2Variant {
  void (*set_basis)(const BasisP2&);
  void (*stage)(const P2Args&, bool, cudaStream_t);
  void (*modal2nodal)(const MeshView&, const double*, double, double, double*, double*, double*, int*,
                      cudaStream_t);
  void (*layout)(bool, const double*, double*, int, int, const int*, cudaStream_t);
  size_t (*tile_smem)(int, int);
};
static const P2Variant kFastP2 = {fast_p2::set_basis_p2, fast_p2::launch_p2_stage, fast_p2::launch_p2_modal2nodal,
                                  fast_p2::launch_p2_layout, fast_p2::p2_tile_smem};
static const P2Variant kStrictP2 = {strict_p2::set_basis_p2, strict_p2::launch_p2_stage,
                                    strict_p2::launch_p2_modal2nodal, strict_p2::launch_p2_layout,
                                    strict_p2::p2_tile_smem};
static const P2Variant kMixedP2 = {mixed_p2::set_basis_p2, mixed_p2::launch_p2_stage,
                                   mixed_p2::launch_p2_modal2nodal, mixed_p2::launch_p2_layout,
                                   mixed_p2::p2_tile_smem};
// the tile plan a p=2 handle's tile kernel runs on: tiles of 64 elements
// (kTileShapes[kP2PlanShape]), the p=2 kernel's tile
constexpr int kP2PlanShape = 1;

}  // namespace dgswem

using namespace dgswem;

struct dgswem_cuda {
  int device = 0;
  const Variant* v = &kFast;
  // per-stage boundary forcing computed on the host (ocean EMO*RFF*COS,
  // flow QNAM*RFF*COS), uploaded once per chunk of steps
  size_t forcing_per_stage = 0;
  int chunk_steps = 0;
  double* forcing_host = nullptr;   // pinned, chunk_steps*nrk*forcing_per_stage
  DevBuf<double> forcing_dev;
  cudaEvent_t forcing_copied = nullptr;
  std::vector<double> emo_h, efa_h, qnam_h, qnph_h;
  int needs = 0, nfeds = 0;
  size_t stage_smem = 0;  // dynamic shared memory of a stage tile
  cudaStream_t stream = nullptr;      // stream the launches go to
  cudaStream_t own_stream = nullptr;  // created with the context
  int ne = 0, np = 0, nrk = 0;
  // scalars kept from the setup
  int nramp = 0, slopeflag = 0, nolifa = 0, nws = 0;
  double dtdp = 0, statim = 0, dramp = 1;
  std::vector<double> atvd, btvd, dtvd;
  std::vector<double> amig, ff, face, per, famig, fff, fface, fper;
  std::vector<char> keep_rhs;  // stage I's RHS is read by a later stage
  Physics ph{};
  MeshView mesh{};
  // device arrays
  DevBuf<double> x, y, dp, hb, egeo, cori, fric, manning, sfac_area, sfac_edge;
  DevBuf<float> egeof;  // FP32 geometry rows of a mixed-precision handle
  DevBuf<int> nm, link, star_ptr, star, ib_elem, ib_led;
  DevBuf<unsigned> einfo, eslot, tile_tasks;
  DevBuf<int> tile_elem_ptr, tile_task_ptr, tile_halo_ptr, tile_halo;
  int ntile = 0;
  // tiles that read no ghost element and no internal-barrier side first
  // (n_tile_interior of them), then the others: the stage can start on the
  // former while the halo exchange that refreshes the ghosts is in flight
  DevBuf<int> tile_order;
  int n_tile_interior = 0;
  // shape of the stage tiles (kTileShapes) and of the limiter blocks
  // (kLimitBlocks): the defaults, or set / picked by dgswem_cuda_autotune
  int tile_shape = kDefaultTileShape, limit_shape = kDefaultLimitShape;
  // modes per variable: 3 (p=1) or 6 (p=2: the p=2 launchers, an edge list of
  // interior edges from the in side and land / ocean edges, and the
  // edge-point flux slots, 36 per element)
  int dofh = 3;
  const P2Variant* v2 = nullptr;
  DevBuf<int> p2_edges;
  DevBuf<double> p2_ef;
  int p2_nedge = 0;
  // the p=2 stage runs as the tile kernel (p2_tile) when its shared memory
  // fits, else as the edge + element kernel pair through p2_ef
  bool p2_tiled = false;
  DevBuf<double> emo_dg, efa_dg, qnam_dg, qnph_dg, ebht, ebcfsp, ibht, ibcfsb, ibcfsp;
  DevBuf<double> wsx, wsy, pr, minmax, staging;
  std::vector<DevBuf<double>> q;    // nrk+1 stage buffers, 9*NE each
  std::vector<DevBuf<double>> rhs;  // nrk RHS buffers (allocated when kept)
  DevBuf<double> ib_rhs;  // internal-barrier terms of the current stage
  DevBuf<int> wd, nodecode, wd_staging;
  DevBuf<int> perm, inv;  // device element order: perm[new] = input id, inv[input] = new
  DevBuf<int> node_perm;  // device node order: node_perm[new] = input id
  std::vector<int> node_perm_h, perm_h;
  // partition (a single one for dgswem_cuda_create): local = owned + ghosts
  int nparts = 1, part = 0, n_own = 0, ne_glob = 0, np_glob = 0;
  // halo index lists (local element ids) per kind and peer: send then receive
  DevBuf<int> halo_idx;
  std::vector<size_t> halo_off[2][2];  // [kind][send 0 / recv 1][peer..peer+1]
  DevBuf<unsigned> err;
  long long launches = 0;
  // per-kernel event timing (dgswem_cuda_profile)
  bool prof_on = false;
  std::vector<cudaEvent_t> ev_pool;
  struct Pending { int kind; cudaEvent_t a, b; };
  std::vector<Pending> pending;
  double prof_ms[4] = {0, 0, 0, 0};
  long long prof_n[4] = {0, 0, 0, 0};
  // discrete adjoint (dgswem_cuda_adjoint_*): lam[I-1] / nu[I-1] the
  // cotangents of stage state I and of its right-hand side; lam[nrk] the
  // current one (of the state the last adjoint step started from)
  int nreds = 0;
  std::vector<DevBuf<double>> adj_lam, adj_nu;
  DevBuf<double> adj_gn, adj_ghb, adj_eb;
  DevBuf<int> adj_edges;  // (element, local edge): interior edges from the in side, land / ocean edges
  int adj_nedge = 0;
  bool adj_on = false;
  // stage states and stage forcing of the steps of one checkpoint segment
  // (dgswem_cuda_adjoint_sweep)
  std::vector<DevBuf<double>> adj_stage;
  DevBuf<double> adj_forc;
  // limiter reverse mode: pre-limiter stage outputs (segment: every x NRK;
  // step-wise: NRK), node bounds / their elements, bound cotangents
  std::vector<DevBuf<double>> adj_pre, adj_pre_step;
  DevBuf<double> adj_mm, adj_lb, adj_nb;
  DevBuf<int> adj_arg;
  // when set, launch_stage copies each stage kernel's output (before the
  // limiter) to keep_pre[irk - 1]
  double* const* keep_pre = nullptr;
  // when set, launch_stage copies WDFLG as each stage kernel reads it to
  // keep_wd[irk - 1]
  int* const* keep_wd = nullptr;
  std::vector<DevBuf<int>> adj_wd, adj_wd_step;  // per segment step x NRK / per NRK
  // gauges: device element, ZE basis values, values / weights; grouped by
  // element (CSR over distinct elements, gauges in input order) for the seed
  int ngauge = 0, ngroup = 0;
  DevBuf<int> gauge_elem, group_elem, group_ptr, group_gauge;
  DevBuf<double> gauge_phi, gauge_val, eta_rec, w_rec;
  // state slots of dgswem_cuda_state_save / _load (checkpoints)
  std::vector<DevBuf<double>> slot_q;
  std::vector<DevBuf<int>> slot_wd;
  // CUDA graphs of graph_steps steps (dgswem_cuda_set_graph): two graphs
  // that differ only in the pinned buffer their first node copies the
  // chunk's stage forcing and ramps from, so that the host fills one while
  // the other runs
  // fort.22 of NWS = 1 read by the handle before every RK stage
  // (dgswem_cuda_met_file): the reader, one block in input node order, and
  // two pinned blocks in device node order, each free again once its event
  // has completed
  dgswem_met_reader* met = nullptr;
  std::vector<double> met_in;
  double* met_pin[2] = {nullptr, nullptr};
  cudaEvent_t met_done[2] = {nullptr, nullptr};
  int met_next = 0;
  int graph_steps = 0, graph_next = 0;
  bool graph_ready = false;
  cudaGraph_t graph[2] = {nullptr, nullptr};
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  double* gbuf_host[2] = {nullptr, nullptr};
  size_t gbuf_bytes = 0;
  cudaEvent_t gdone[2] = {nullptr, nullptr};
  DevBuf<double> gbuf_dev;
  double* graph_q0 = nullptr;      // buffer that held the state at capture
  long long graph_launches = 0;    // kernels per graph
};

namespace {

// Entry points of the p=1 path only (the limiter and its reverse mode, the
// adjoint, state slots, partitions, tile shapes, graphs)
void need_p1(const dgswem_cuda* h, const char* what) {
  if (h && h->dofh != 3) throw Failure(DGSWEM_ERR_ARG, std::string(what) + " is p=1 only");
}

void check_launch(dgswem_cuda* h, const char* what = "kernel") {
  ++h->launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Failure(DGSWEM_ERR_CUDA, std::string("launch of ") + what + ": " + cudaGetErrorString(e));
}

cudaEvent_t take_event(dgswem_cuda* h) {
  if (!h->ev_pool.empty()) {
    cudaEvent_t e = h->ev_pool.back();
    h->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  DG_CUDA(cudaEventCreate(&e));
  return e;
}

void prof_flush(dgswem_cuda* h) {
  if (h->pending.empty()) return;
  DG_CUDA(cudaStreamSynchronize(h->stream));
  for (auto& p : h->pending) {
    float ms = 0.f;
    DG_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
    h->prof_ms[p.kind] += ms;
    h->prof_n[p.kind] += 1;
    h->ev_pool.push_back(p.a);
    h->ev_pool.push_back(p.b);
  }
  h->pending.clear();
}

// Records CUDA events around one launch on the launching stream when
// profiling is on.
struct LaunchTimer {
  dgswem_cuda* h;
  int kind;
  cudaEvent_t a = nullptr;
  static constexpr const char* kNames[4] = {"stage_p1", "node_minmax", "limit_wetdry", "other"};
  LaunchTimer(dgswem_cuda* hh, int k) : h(hh), kind(k) {
    if (h->prof_on) {
      a = take_event(h);
      DG_CUDA(cudaEventRecord(a, h->stream));
    }
  }
  void done() {
    check_launch(h, kNames[kind]);
    if (a) {
      cudaEvent_t b = take_event(h);
      DG_CUDA(cudaEventRecord(b, h->stream));
      h->pending.push_back({kind, a, b});
      if (h->pending.size() > 2048) prof_flush(h);
    }
  }
};

unsigned grid_for(int n, int block) { return (unsigned)((n + block - 1) / block); }

// Stage tile plan of the handle's tile shape (h->tile_shape): for each tile
// of consecutive elements, the edge tasks it evaluates and the out-of-tile
// neighbours (halo) they read.  Edge ownership: a boundary edge of a listed
// kind and an internal-barrier side belong to their element; an interior
// edge inside the tile is evaluated once, by its in side NEDEL(1); an
// interior edge to another tile is evaluated by both tiles, each for its own
// element, in the reference's in/ex orientation.  Tasks: interior edges in
// element order, then the boundary kinds grouped, so that a warp's tasks
// mostly take one branch.  Tiles cover the first n_tiled elements (the owned
// ones); `ne` is the row stride of link (all local elements, ghosts
// included).  Tiles are cut sequentially, then planned in parallel (each
// writes only its own elements' eslot).
void build_tile_plan(dgswem_cuda* h, int n_tiled, int ne, const std::vector<int>& link,
                     const std::vector<unsigned>& einfo) {
  const TileShape shape = kTileShapes[h->tile_shape];
  // Tiles: consecutive elements, at most shape.tile of them and at most
  // shape.threads edge tasks (one pass of the block over its tasks).  An
  // element adds a task per listed boundary edge and per interior edge whose
  // neighbour is not already in the tile.
  std::vector<int> elem_ptr(1, 0);
  {
    int t0 = 0, count = 0;
    for (int e = 0; e < n_tiled; ++e) {
      int add = 0;
      for (int l = 0; l < 3; ++l) {
        const unsigned kind = ei_kind(einfo[e], l);
        if (kind == kNone) continue;
        if (kind == kInterior) {
          const int nb = link[(size_t)l * ne + e];
          if (nb >= t0 && nb < e) continue;
        }
        ++add;
      }
      if (e - t0 == shape.tile || count + add > shape.threads) {
        elem_ptr.push_back(e);
        t0 = e;
        count = 0;
        e -= 1;  // recount the element against the new tile
        continue;
      }
      count += add;
    }
    elem_ptr.push_back(n_tiled);
  }
  const int ntile = (int)elem_ptr.size() - 1;
  std::vector<std::vector<unsigned>> ttasks(ntile);  // (word, list) pairs per tile
  std::vector<std::vector<int>> thalo(ntile);
  std::vector<unsigned> eslot(ne, 0u);
  int max_halo = 0, max_tasks = 0;
  struct Task {
    unsigned word, list;
    int el, led;
  };
#pragma omp parallel
  {
    std::vector<int> hl;
    std::vector<Task> tt;
#pragma omp for schedule(dynamic, 64) reduction(max : max_halo, max_tasks)
    for (int t = 0; t < ntile; ++t) {
      const int t0 = elem_ptr[t], t1 = elem_ptr[t + 1];
      hl.clear();
      for (int e = t0; e < t1; ++e)
        for (int l = 0; l < 3; ++l)
          if (ei_kind(einfo[e], l) == kInterior) {
            const int nb = link[(size_t)l * ne + e];
            if (nb < t0 || nb >= t1) hl.push_back(nb);
          }
      std::sort(hl.begin(), hl.end());
      hl.erase(std::unique(hl.begin(), hl.end()), hl.end());
      auto slot = [&](int g) -> unsigned {
        if (g >= t0 && g < t1) return (unsigned)(g - t0);
        return (unsigned)(shape.tile + (std::lower_bound(hl.begin(), hl.end(), g) - hl.begin()));
      };
      tt.clear();
      for (int pass = 0; pass < 2; ++pass)  // interior edges, then boundary kinds
        for (unsigned want = pass == 0 ? (unsigned)kInterior : 1u; want <= (pass == 0 ? 0u : 6u); ++want)
          for (int e = t0; e < t1; ++e)
            for (int l = 0; l < 3; ++l) {
              const unsigned info = einfo[e], kind = ei_kind(info, l);
              if (kind != want) continue;
              const int lk = link[(size_t)l * ne + e];
              unsigned w = kind << TaskBits::kKind, list = 0;
              if (kind == kInterior) {
                const bool local = lk >= t0 && lk < t1, in_side = ei_flag(info, l) != 0;
                if (local && !in_side) continue;  // the in side's task
                const unsigned nled = ei_nled(info, l);
                if (in_side)
                  w |= (unsigned)l << TaskBits::kLedIn | nled << TaskBits::kLedEx | slot(e) << TaskBits::kInSlot |
                       slot(lk) << TaskBits::kExSlot;
                else
                  w |= nled << TaskBits::kLedIn | (unsigned)l << TaskBits::kLedEx | 1u << TaskBits::kFlip |
                       slot(lk) << TaskBits::kInSlot | slot(e) << TaskBits::kExSlot;
              } else {
                w |= (unsigned)l << TaskBits::kLedIn | slot(e) << TaskBits::kInSlot;
                list = kind == kIBarrier ? (unsigned)lk * 2u + (ei_flag(info, l) ? 0u : 1u) : (unsigned)lk;
              }
              tt.push_back({w, list, e, l});
            }
      for (int e = t0; e < t1; ++e) eslot[e] = kNoTask | kNoTask << 10 | kNoTask << 20;
      auto set_slot = [&](int e, int l, unsigned ti) {
        eslot[e] = (eslot[e] & ~(kNoTask << (10 * l))) | ti << (10 * l);
      };
      for (size_t i = 0; i < tt.size(); ++i) set_slot(tt[i].el, tt[i].led, (unsigned)i);
      for (int e = t0; e < t1; ++e)  // shared edges inside the tile: the in side's task
        for (int l = 0; l < 3; ++l) {
          const unsigned info = einfo[e];
          if (ei_kind(info, l) != kInterior || ei_flag(info, l)) continue;
          const int nb = link[(size_t)l * ne + e];
          if (nb < t0 || nb >= t1) continue;
          set_slot(e, l, (eslot[nb] >> (10 * ei_nled(info, l))) & kNoTask);
        }
      std::vector<unsigned>& out = ttasks[t];
      out.reserve(2 * tt.size());
      for (const Task& k : tt) {
        out.push_back(k.word);
        out.push_back(k.list);
      }
      thalo[t] = hl;
      max_halo = std::max(max_halo, (int)hl.size());
      max_tasks = std::max(max_tasks, (int)tt.size());
    }
  }
  if (max_halo + shape.tile > kMaxTileSlots || max_tasks >= (int)kNoTask)
    throw Failure(DGSWEM_ERR_ARG, "stage tile plan exceeds the task word's slot range");
  const size_t stage_smem = stage_layout(shape.tile, max_halo, std::max(max_tasks, 1), h->v->real_bytes).bytes;
  int dev_smem = 0;
  DG_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
  if (stage_smem > (size_t)dev_smem)
    throw Failure(DGSWEM_ERR_ARG, "stage tile needs " + std::to_string(stage_smem) +
                                      " bytes of shared memory, the device allows " + std::to_string(dev_smem));
  std::vector<int> task_ptr(ntile + 1, 0), halo_ptr(ntile + 1, 0), halo;
  std::vector<unsigned> tasks;
  for (int t = 0; t < ntile; ++t) {
    task_ptr[t + 1] = task_ptr[t] + (int)ttasks[t].size() / 2;
    halo_ptr[t + 1] = halo_ptr[t] + (int)thalo[t].size();
  }
  tasks.reserve(2 * (size_t)task_ptr[ntile]);
  halo.reserve((size_t)halo_ptr[ntile]);
  for (int t = 0; t < ntile; ++t) {
    tasks.insert(tasks.end(), ttasks[t].begin(), ttasks[t].end());
    halo.insert(halo.end(), thalo[t].begin(), thalo[t].end());
  }
  {
    std::vector<int> order, rest;
    for (int t = 0; t < ntile; ++t) {
      bool interior = true;
      for (int g : thalo[t]) interior = interior && g < n_tiled;
      for (size_t i = 0; i < ttasks[t].size(); i += 2)
        interior = interior && (ttasks[t][i] & 7u) != kIBarrier;
      (interior ? order : rest).push_back(t);
    }
    h->n_tile_interior = (int)order.size();
    order.insert(order.end(), rest.begin(), rest.end());
    h->tile_order.upload(order.empty() ? std::vector<int>(1, 0) : order);
  }
  h->ntile = ntile;
  h->tile_elem_ptr.upload(elem_ptr);
  h->tile_task_ptr.upload(task_ptr);
  h->tile_halo_ptr.upload(halo_ptr);
  h->tile_tasks.upload(tasks.empty() ? std::vector<unsigned>(2, 0u) : tasks);
  h->tile_halo.upload(halo.empty() ? std::vector<int>(1, 0) : halo);
  h->eslot.upload(eslot);
  h->stage_smem = stage_smem;
  MeshView& m = h->mesh;
  m.max_halo = max_halo;
  m.max_tasks = max_tasks;
  m.tile_elem_ptr = h->tile_elem_ptr.p;
  m.tile_task_ptr = h->tile_task_ptr.p;
  m.tile_tasks = reinterpret_cast<const uint2*>(h->tile_tasks.p);
  m.tile_halo_ptr = h->tile_halo_ptr.p;
  m.tile_halo = h->tile_halo.p;
  m.eslot = h->eslot.p;
}

// Device element and node order: elements sorted along a Morton (Z-order)
// curve of their centroids, nodes along the same curve of their coordinates
// (stable sorts, ties keep the input order).  A stage tile of consecutive
// elements is then a compact patch of the mesh with a short perimeter -- few
// edges to other tiles, a small halo -- and the nodes an element touches lie
// close together in memory.  perm[local] = input index.  Nothing in the
// arithmetic depends on the numbering: edge orientation (NEDEL), the
// interior-edge order (edge numbers) and the node stars (built in input
// element order) are those of the input mesh.  A partitioned handle keeps
// its owned elements (a contiguous range of the global Morton order) first,
// then its ghost elements (partition.h).
void build_layout(dgswem_cuda* h, const dgswem_cuda_setup* s, const PartPlan& plan) {
  const int ne = s->ne, np = s->np, ned = s->nedges;
  auto need = [](bool ok, const char* what) {
    if (!ok) throw Failure(DGSWEM_ERR_ARG, what);
  };
  need(s->nm && s->x && s->y && s->dp && s->neled && s->nedel && s->nedsd && s->hb, "setup lacks mesh arrays");
  need(s->ze && s->qx && s->qy && s->wdflg, "setup lacks the initial state");
  need(s->atvd && s->btvd && s->dtvd, "setup lacks RK tables");
  // local elements (owned, then ghosts) and the nodes they touch
  const std::vector<int>& perm = plan.local;
  const int nl = (int)perm.size(), n_own = plan.n_own;
  std::vector<int> inv(ne, -1);
  for (int i = 0; i < nl; ++i) inv[perm[i]] = i;
  std::vector<int> node_perm, node_inv(np, -1);
  {
    std::vector<char> used(np, 0);
    for (int i = 0; i < nl; ++i)
      for (int v = 0; v < 3; ++v) used[s->nm[perm[i] + (size_t)ne * v] - 1] = 1;
    std::vector<int> ncomp;
    mesh_components(s, &ncomp);
    const std::vector<int> norder =
        morton_order(std::vector<double>(s->x, s->x + np), std::vector<double>(s->y, s->y + np), ncomp);
    for (int n : norder)
      if (used[n]) node_perm.push_back(n);
  }
  const int npl = (int)node_perm.size();
  for (int i = 0; i < npl; ++i) node_inv[node_perm[i]] = i;
  // nodal arrays in the device node order
  auto node_permuted = [&](const double* a) {
    std::vector<double> out(npl);
    for (int i = 0; i < npl; ++i) out[i] = a[node_perm[i]];
    return out;
  };
  const std::vector<double> xd = node_permuted(s->x), yd = node_permuted(s->y);
  std::vector<int> nm(3 * (size_t)nl);
  for (int i = 0; i < nl; ++i)
    for (int v = 0; v < 3; ++v) nm[(size_t)v * nl + i] = node_inv[s->nm[perm[i] + (size_t)ne * v] - 1];
  // boundary membership of each edge: kind, list index, side
  std::vector<int> bkind(ned + 1, -1), bidx(ned + 1, -1), bside(ned + 1, 0);
  auto mark = [&](const int* list, int n, unsigned kind) {
    for (int i = 0; i < n; ++i) {
      int g = list[i];
      need(g >= 1 && g <= ned, "boundary edge list refers to a missing edge");
      need(bkind[g] < 0, "an edge appears in more than one boundary list");
      bkind[g] = (int)kind;
      bidx[g] = i;
    }
  };
  if (s->needs) mark(s->needn, s->needs, kOcean);
  if (s->nleds) mark(s->nledn, s->nleds, kLand);
  if (s->nfeds) mark(s->nfedn, s->nfeds, kFlow);
  if (s->nreds) mark(s->nredn, s->nreds, kRadiation);
  if (s->nebseg) mark(s->nebsegn, s->nebseg, kEBarrier);
  std::vector<int> ib_elem(2 * (size_t)std::max(s->nibseg, 1), -1), ib_led(2 * (size_t)std::max(s->nibseg, 1), 0);
  for (int L = 0; L < s->nibseg; ++L) {
    int gb = s->nibsegn[2 * L], gf = s->nibsegn[2 * L + 1];
    if (gf == 0) continue;  // no opposite edge: the reference skips the segment
    for (int side = 0; side < 2; ++side) {
      int g = side == 0 ? gb : gf;
      need(g >= 1 && g <= ned, "NIBSEGN refers to a missing edge");
      need(bkind[g] < 0, "a barrier edge appears in more than one boundary list");
      bkind[g] = kIBarrier;
      bidx[g] = L;
      bside[g] = side;
      ib_elem[2 * L + side] = inv[s->nedel[2 * (size_t)(g - 1)] - 1];
      ib_led[2 * L + side] = s->nedsd[2 * (size_t)(g - 1)] - 1;
    }
    if (ib_elem[2 * L] < 0 || ib_elem[2 * L + 1] < 0) ib_elem[2 * L] = ib_elem[2 * L + 1] = -1;  // not local
  }
  std::vector<int> link(3 * (size_t)nl, -1);
  std::vector<unsigned> einfo(nl, 0u);
  for (int i = 0; i < nl; ++i) {
    const int e = perm[i];
    unsigned info = 0u;
    std::array<std::pair<long long, int>, 3> key;
    for (int l = 0; l < 3; ++l) {
      int g = s->neled[l + 3 * (size_t)e];
      need(g >= 1 && g <= ned, "NELED refers to a missing edge");
      int a = s->nedel[2 * (size_t)(g - 1)], b = s->nedel[2 * (size_t)(g - 1) + 1];
      unsigned kind, flag = 0, nled = 0;
      int lk;
      if (a != 0 && b != 0) {
        need(bkind[g] < 0, "an interior edge also appears in a boundary list");
        bool first = a == e + 1;
        need(first || b == e + 1, "NEDEL does not contain the element of NELED");
        kind = kInterior;
        flag = first ? 1u : 0u;
        lk = inv[(first ? b : a) - 1];
        nled = (unsigned)(s->nedsd[2 * (size_t)(g - 1) + (first ? 1 : 0)] - 1);
        key[l] = {(long long)8 << 40 | g, l};  // interior edges last, in edge-number order
        if (lk < 0) {  // a ghost's neighbour outside the partition: never evaluated
          need(i >= n_own, "partition halo lacks an edge neighbour of an owned element");
          kind = kNone;
          flag = 0;
          nled = 0;
        }
      } else if (bkind[g] >= 0) {
        kind = (unsigned)bkind[g];
        lk = bidx[g];
        if (kind == kIBarrier) flag = bside[g] == 0 ? 1u : 0u;
        key[l] = {(long long)kind << 40 | (long long)lk << 1 | (flag ? 0 : 1), l};
      } else {
        kind = kNone;
        lk = -1;
        key[l] = {(long long)9 << 40, l};
      }
      link[(size_t)l * nl + i] = lk;
      info |= kind << (3 * l);
      info |= flag << (9 + l);
      info |= (nled & 3u) << (12 + 2 * l);
    }
    std::sort(key.begin(), key.end());
    for (int slot = 0; slot < 3; ++slot) info |= (unsigned)key[slot].second << (18 + 2 * slot);
    einfo[i] = info;
  }
  build_tile_plan(h, n_own, nl, link, einfo);
  // node -> element star in the input element order (the order of the
  // reference's loops over elements), holding device element ids; complete
  // for every node of an owned element
  std::vector<int> sp(npl + 1, 0), st(3 * (size_t)nl);
  for (int i = 0; i < nl; ++i)
    for (int v = 0; v < 3; ++v) ++sp[nm[(size_t)v * nl + i] + 1];
  for (int n = 0; n < npl; ++n) sp[n + 1] += sp[n];
  {
    std::vector<int> cur(sp.begin(), sp.end() - 1);
    for (int e = 0; e < ne; ++e) {
      const int i = inv[e];
      if (i < 0) continue;
      for (int v = 0; v < 3; ++v) st[cur[nm[(size_t)v * nl + i]]++] = i;
    }
  }
  h->perm.upload(perm);
  h->inv.upload(inv);
  h->perm_h = perm;
  h->nm.upload(nm);
  h->link.upload(link);
  h->einfo.upload(einfo);
  h->star_ptr.upload(sp);
  h->star.upload(st);
  h->ib_elem.upload(ib_elem);
  h->ib_led.upload(ib_led);
  h->node_perm.upload(node_perm);
  h->node_perm_h = node_perm;
  h->x.upload(xd);
  h->y.upload(yd);
  h->dp.upload(node_permuted(s->dp));
  std::vector<double> hb((size_t)h->dofh * nl);
  for (int i = 0; i < nl; ++i)
    for (int k = 0; k < h->dofh; ++k) hb[(size_t)k * nl + i] = s->hb[k + (size_t)s->dofh * perm[i]];
  h->hb.upload(hb);
  // per-element coefficients: a scalar when uniform
  auto uniform = [&](const double* a, double* val) {
    if (!a) { *val = 0.0; return true; }
    for (int e = 1; e < ne; ++e)
      if (a[e] != a[0]) return false;
    *val = a[0];
    return true;
  };
  double c0 = 0.0, f0 = s->cf;
  auto permuted = [&](const double* a) {
    std::vector<double> out(nl);
    for (int i = 0; i < nl; ++i) out[i] = a[perm[i]];
    return out;
  };
  if (!uniform(s->cori_el, &c0)) h->cori.upload(permuted(s->cori_el));
  if (!uniform(s->fric_el, &f0)) h->fric.upload(permuted(s->fric_el));
  h->ph.cori = c0;
  h->ph.fric = f0;
  if (s->load_manning) {
    need(s->manning != nullptr, "load_manning set without ManningsN");
    h->manning.upload(node_permuted(s->manning));
  }
  // element geometry table (EGeo rows): the reference's formulas evaluated
  // once, in the same order as the oracle, instead of every stage
  {
    std::vector<double> eg((size_t)EGeo::kRows * nl, 0.0);
    auto at = [&](int r, int e) -> double& { return eg[(size_t)r * nl + e]; };
#pragma omp parallel for schedule(static)
    for (int e = 0; e < nl; ++e) {
      double xs[3], ys[3];
      for (int v = 0; v < 3; ++v) {
        xs[v] = xd[nm[(size_t)v * nl + e]];
        ys[v] = yd[nm[(size_t)v * nl + e]];
      }
      const double areas = (xs[0] - xs[2]) * (ys[1] - ys[2]) + (xs[2] - xs[1]) * (ys[0] - ys[2]);
      at(EGeo::kAreas, e) = areas;
      for (int l = 0; l < 3; ++l) {
        const int a = (l + 1) % 3, b = (l + 2) % 3;
        const double dy = ys[b] - ys[a], dx = xs[b] - xs[a];
        const double len = std::sqrt(dy * dy + dx * dx);
        at(EGeo::kXlen + l, e) = len;
        at(EGeo::kNx + l, e) = (ys[b] - ys[a]) / len;
        at(EGeo::kNy + l, e) = -(xs[b] - xs[a]) / len;
      }
      for (int l = 0; l < 3; ++l) at(EGeo::kEdfac + l, e) = at(EGeo::kXlen + l, e) / areas;
      const double area = areas * 0.5;
      at(EGeo::kDrdx, e) = 1.0 / area * (ys[2] - ys[0]);
      at(EGeo::kDsdx, e) = 1.0 / area * (ys[0] - ys[1]);
      at(EGeo::kDrdy, e) = 1.0 / area * (xs[0] - xs[2]);
      at(EGeo::kDsdy, e) = 1.0 / area * (xs[1] - xs[0]);
      if (s->load_manning)
        at(EGeo::kNbar, e) = (s->manning[node_perm[nm[e]]] + s->manning[node_perm[nm[(size_t)nl + e]]] +
                              s->manning[node_perm[nm[(size_t)2 * nl + e]]]) / 3.;
    }
    h->egeo.upload(eg);
    if (h->v->real_bytes == 4) h->egeof.upload(std::vector<float>(eg.begin(), eg.end()));
  }
  if (s->ics == 2) {  // SFAC_ELEM / SFACED (prep_DG.F:1055-1100), host cos
    const BasisP1 B = make_basis_p1();
    const double R = 6378206.4;
    std::vector<double> sa(3 * (size_t)nl), se(9 * (size_t)nl);
    for (int e = 0; e < nl; ++e) {
      const double y1 = yd[nm[e]], y2 = yd[nm[(size_t)nl + e]], y3 = yd[nm[(size_t)2 * nl + e]];
      const double yd[3] = {1.0 / 3.0 * (y1 + y2 + y3), -(1.0 / 6.0 * (y1 + y2)) + 1.0 / 3.0 * y3,
                            -(0.5 * y1) + 0.5 * y2};
      for (int i = 0; i < 3; ++i) {
        double yel = 0.0;
        for (int k = 0; k < 3; ++k) yel = yel + yd[k] * B.phi_area[k][i];
        sa[(size_t)i * nl + e] = std::cos(s->sfea0) / std::cos(yel / R);
      }
      for (int l = 0; l < 3; ++l)
        for (int i = 0; i < 3; ++i) {
          double yed = 0.0;
          for (int k = 0; k < 3; ++k) yed = yed + yd[k] * B.phi_edge[l][i][k];
          se[(size_t)(l * 3 + i) * nl + e] = std::cos(s->sfea0) / std::cos(yed / R);
        }
    }
    h->sfac_area.upload(sa);
    h->sfac_edge.upload(se);
  }
  // boundary forcing tables (copied in the reference's Fortran layout)
  const int nbfr = s->nbfr, nffr = s->nffr;
  if (s->needs && nbfr) {
    h->amig.assign(s->amig, s->amig + nbfr);
    h->ff.assign(s->ff, s->ff + nbfr);
    h->face.assign(s->face, s->face + nbfr);
    h->per.assign(s->per, s->per + nbfr);
  }
  if (s->nfeds && nffr) {
    h->famig.assign(s->famig, s->famig + nffr);
    h->fff.assign(s->fff, s->fff + nffr);
    h->fface.assign(s->fface, s->fface + nffr);
    h->fper.assign(s->fper, s->fper + nffr);
  }
  if (s->nebseg) {
    h->ebht.upload(std::vector<double>(s->ebht, s->ebht + s->nebseg));
    h->ebcfsp.upload(std::vector<double>(s->ebcfsp, s->ebcfsp + s->nebseg));
  }
  if (s->nibseg) {
    h->ibht.upload(std::vector<double>(s->ibht, s->ibht + s->nibseg));
    h->ibcfsb.upload(std::vector<double>(s->ibcfsb, s->ibcfsb + s->nibseg));
    h->ibcfsp.upload(std::vector<double>(s->ibcfsp, s->ibcfsp + s->nibseg));
    h->ib_rhs.alloc(18 * (size_t)s->nibseg);
  }
  MeshView& m = h->mesh;
  m.ne = nl;
  m.np = npl;
  h->ne = nl;
  h->np = npl;
  h->n_own = n_own;
  h->ne_glob = ne;
  h->np_glob = np;
  h->nparts = plan.nparts;
  h->part = plan.part;
  m.x = h->x.p; m.y = h->y.p; m.dp = h->dp.p; m.nm = h->nm.p; m.link = h->link.p; m.einfo = h->einfo.p;
  m.hb = h->hb.p; m.egeo = h->egeo.p; m.egeof = h->egeof.p; m.cori = h->cori.p; m.fric = h->fric.p; m.manning = h->manning.p;
  m.sfac_area = h->sfac_area.p; m.sfac_edge = h->sfac_edge.p;
  m.star_ptr = h->star_ptr.p; m.star = h->star.p; m.node_perm = h->node_perm.p;
  m.needs = s->needs; m.nfeds = s->nfeds; m.nebseg = s->nebseg; m.nibseg = s->nibseg;
  m.nbfr = h->amig.empty() ? 0 : nbfr;
  m.nffr = h->famig.empty() ? 0 : nffr;
  m.emo_dg = h->emo_dg.p; m.efa_dg = h->efa_dg.p; m.qnam_dg = h->qnam_dg.p; m.qnph_dg = h->qnph_dg.p;
  m.ebht = h->ebht.p; m.ebcfsp = h->ebcfsp.p;
  m.ib_elem = h->ib_elem.p; m.ib_led = h->ib_led.p;
  m.ibht = h->ibht.p; m.ibcfsb = h->ibcfsb.p; m.ibcfsp = h->ibcfsp.p;
}

// Halo index lists of a partitioned handle (local element ids), per kind,
// send lists then receive lists, peer by peer (partition.h).
void build_halo(dgswem_cuda* h, const dgswem_cuda_setup* s, const PartPlan& plan) {
  std::vector<int> inv(s->ne, -1);
  for (size_t i = 0; i < plan.local.size(); ++i) inv[plan.local[i]] = (int)i;
  std::vector<int> idx;
  for (int k = 0; k < 2; ++k)
    for (int dir = 0; dir < 2; ++dir) {
      auto& off = h->halo_off[k][dir];
      off.assign(1, idx.size());
      const auto& lists = dir == 0 ? plan.send[k] : plan.recv[k];
      for (int q = 0; q < plan.nparts; ++q) {
        for (int e : lists[q]) {
          const int i = inv[e];
          if (i < 0 || (dir == 0) != (i < plan.n_own))
            throw Failure(DGSWEM_ERR_ARG, "partition halo list refers to an element of the wrong kind");
          idx.push_back(i);
        }
        off.push_back(idx.size());
      }
    }
  h->halo_idx.upload(idx.empty() ? std::vector<int>(1, 0) : idx);
}

// Host state (Fortran layout, input element order, all NE elements) -> the
// local elements' device state (stage buffer 1) and WDFLG.
void upload_state(dgswem_cuda* h, const double* ze, const double* qx, const double* qy, const int* wdflg) {
  const int nl = h->ne, ng = h->ne_glob;
  const size_t dofh = (size_t)h->dofh;
  h->staging.ensure(dofh * ng);
  const double* src[3] = {ze, qx, qy};
  for (int var = 0; var < 3; ++var) {
    if (!src[var]) continue;
    DG_CUDA(cudaMemcpyAsync(h->staging.p, src[var], dofh * ng * sizeof(double), cudaMemcpyHostToDevice,
                            h->stream));
    if (h->v2)
      h->v2->layout(true, h->staging.p, h->q[0].p, nl, var, h->perm.p, h->stream);
    else
      h->v->f2s(h->staging.p, h->q[0].p, nl, var, h->perm.p, grid_for(nl, kPointBlock), h->stream);
    check_launch(h, "fortran_to_soa");
  }
  if (wdflg) {
    DG_CUDA(cudaMemcpyAsync(h->wd_staging.p, wdflg, (size_t)ng * sizeof(int), cudaMemcpyHostToDevice, h->stream));
    h->v->gather_int(h->wd_staging.p, h->wd.p, h->perm.p, nl, grid_for(nl, kPointBlock), h->stream);
    check_launch(h, "gather_int");
  }
  DG_CUDA(cudaStreamSynchronize(h->stream));
}

// DG_hydro_timestep.F:79-100: stage time and ramp
void stage_clock(const dgswem_cuda* h, int it, int irk, double* timedg, double* rampdg) {
  const double itdt = it * h->dtdp;
  const double time_a = itdt + h->statim * 86400.0;
  const double dtvd = h->dtvd[irk - 1];
  *timedg = time_a - h->dtdp + dtvd * h->dtdp;
  *rampdg = 1.0;
  if (h->nramp == 1 || h->nramp == 2) *rampdg = std::tanh((2.0 * ((it - 1) + dtvd) * h->dtdp / 86400.0) / h->dramp);
}

// Host part of the boundary forcing of one stage: the ocean harmonic
// endpoint values (ocean_edge_hydro.F:148-177) and the flow boundary normal
// flux terms (flow_edge_hydro.F:108-125), with the host's cos.
void stage_forcing(const dgswem_cuda* h, double timedg, double rampdg, double* out) {
  const int nbfr = (int)h->amig.size(), nffr = (int)h->famig.size();
  const int needs = h->needs, nfeds = h->nfeds;
  for (int f = 0; f < nbfr; ++f) {
    const double ncyc = h->per[f] == 0.0 ? 0.0 : (double)(long long)(timedg / h->per[f]);
    const double argj = h->amig[f] * (timedg - ncyc * h->per[f]) + h->face[f];
    const double rff = h->ff[f] * rampdg;
    for (int l = 0; l < needs; ++l)
      for (int ipt = 0; ipt < 2; ++ipt) {
        const size_t at = f + (size_t)nbfr * (l + (size_t)needs * ipt);
        out[((size_t)f * needs + l) * 2 + ipt] = h->emo_h[at] * rff * std::cos(argj - h->efa_h[at]);
      }
  }
  double* fq = out + (size_t)nbfr * needs * 2;
  const double xegp[3] = {-1.0, 0.0, 1.0};
  for (int f = 0; f < nffr; ++f) {
    const double ncyc = h->fper[f] == 0.0 ? 0.0 : (double)(long long)(timedg / h->fper[f]);
    const double argj = h->famig[f] * (timedg - ncyc * h->fper[f]) + h->fface[f];
    const double rff = h->fff[f] * rampdg;
    for (int l = 0; l < nfeds; ++l) {
      const size_t a0 = f + (size_t)nffr * l, a1 = f + (size_t)nffr * (l + (size_t)nfeds);
      for (int j = 0; j < 3; ++j) {
        const double qa = 0.5 * (h->qnam_h[a0] + h->qnam_h[a1]) + 0.5 * (h->qnam_h[a1] - h->qnam_h[a0]) * xegp[j];
        const double qp = 0.5 * (h->qnph_h[a0] + h->qnph_h[a1]) + 0.5 * (h->qnph_h[a1] - h->qnph_h[a0]) * xegp[j];
        fq[((size_t)f * nfeds + l) * 3 + j] = qa * rff * std::cos(argj - qp);
      }
    }
  }
}

// One RK stage: the stage kernel writes stage buffer irk for the owned
// elements (launch_stage_rhs), then the limiter and WETDRY (launch_limit).
// The p=2 stage: edge kernel, then element kernel (SSP combination included).
void launch_stage_p2(dgswem_cuda* h, int it, int irk, const double* forcing, const double* ramp) {
  const int nrk = h->nrk;
  P2Args A{};
  A.m = h->mesh;
  A.ph = h->ph;
  {
    const Physics& p = h->ph;
    A.pf = PhysF{(float)p.g, (float)p.nleq, (float)p.leq, (float)p.nleqg, (float)p.fg_l, (float)p.tau_cap,
                 (float)p.cori, (float)p.fric, (float)p.cf};
  }
  A.irk = irk;
  A.qin = h->q[irk - 1].p;
  A.qout = h->q[irk].p;
  for (int I = 1; I <= irk; ++I) {
    A.qhist[I - 1] = h->q[I - 1].p;
    A.rhist[I - 1] = h->rhs[I - 1].p;
    A.a[I - 1] = h->atvd[(size_t)(irk - 1) * nrk + (I - 1)];
    A.b[I - 1] = h->btvd[(size_t)(irk - 1) * nrk + (I - 1)] * h->dtdp;
  }
  A.rout = h->keep_rhs[irk - 1] ? h->rhs[irk - 1].p : nullptr;
  double timedg;
  stage_clock(h, it, irk, &timedg, &A.rampdg);
  A.ramp = ramp;
  A.ocean_zg = forcing;
  A.wsx = h->wsx.p;
  A.wsy = h->wsy.p;
  A.pr = h->pr.p;
  A.ef = h->p2_ef.p;
  A.edges = h->p2_edges.p;
  A.nedge = h->p2_nedge;
  A.ne_act = h->n_own;
  A.err = h->err.p;
  A.ntile = h->p2_tiled ? h->ntile : 0;
  const bool nonlin = h->ph.nleq == 1.0 && h->ph.leq == 0.0;
  LaunchTimer t(h, 0);
  h->v2->stage(A, nonlin, h->stream);
  if (!A.ntile) ++h->launches;  // the edge + element kernel pair
  t.done();
}

// Tiles of a stage launch (dgswem_cuda_stage_rhs_tiles): all, those that read
// no ghost (interior), or the others (boundary)
enum TileSet { kAllTiles = 0, kInteriorTiles = 1, kBoundaryTiles = 2 };

void launch_stage_rhs(dgswem_cuda* h, int it, int irk, const double* forcing, const double* ramp = nullptr,
                      TileSet set = kAllTiles) {
  if (h->v2) {
    launch_stage_p2(h, it, irk, forcing, ramp);
    return;
  }
  const int nrk = h->nrk;
  StageArgs A{};
  A.m = h->mesh;
  A.ph = h->ph;
  {
    const Physics& p = h->ph;
    A.pf = PhysF{(float)p.g, (float)p.nleq, (float)p.leq, (float)p.nleqg, (float)p.fg_l, (float)p.tau_cap,
                 (float)p.cori, (float)p.fric, (float)p.cf};
  }
  A.irk = irk;
  A.qin = h->q[irk - 1].p;
  A.qout = h->q[irk].p;
  for (int I = 1; I <= irk; ++I) {
    A.qhist[I - 1] = h->q[I - 1].p;
    A.rhist[I - 1] = h->rhs[I - 1].p;
    A.a[I - 1] = h->atvd[(size_t)(irk - 1) * nrk + (I - 1)];
    A.b[I - 1] = h->btvd[(size_t)(irk - 1) * nrk + (I - 1)] * h->dtdp;
  }
  A.rout = h->keep_rhs[irk - 1] ? h->rhs[irk - 1].p : nullptr;
  A.wd = h->wd.p;
  stage_clock(h, it, irk, &A.timedg, &A.rampdg);
  A.ramp = ramp;
  A.ocean_zg = forcing;
  A.flow_qn = forcing ? forcing + (size_t)h->amig.size() * h->needs * 2 : nullptr;
  A.wsx = h->wsx.p;
  A.wsy = h->wsy.p;
  A.pr = h->pr.p;
  A.ib_rhs = h->ib_rhs.p;
  A.err = h->err.p;
  const bool nonlin = h->ph.nleq == 1.0 && h->ph.leq == 0.0;
  if (h->mesh.nibseg > 0 && set != kInteriorTiles) {  // interior tiles have no barrier sides
    LaunchTimer t(h, 3);
    h->v->ibarrier(A, nonlin, h->stream);
    t.done();
  }
  unsigned grid = (unsigned)h->ntile;
  if (set != kAllTiles) {
    A.tile_list = h->tile_order.p;
    A.tile_off = set == kInteriorTiles ? 0 : h->n_tile_interior;
    grid = set == kInteriorTiles ? (unsigned)h->n_tile_interior : (unsigned)(h->ntile - h->n_tile_interior);
  }
  if (grid > 0) {
    LaunchTimer t(h, 0);
    h->v->stage(A, nonlin, h->tile_shape, grid, h->stage_smem, h->stream);
    t.done();
  }
}

// SLOPELIMITER5 and WETDRY on stage buffer irk (owned elements)
void launch_limit(dgswem_cuda* h, int irk) {
  if (h->v2) return;  // neither limiter nor WETDRY at p=2
  const bool wetdry = h->nolifa >= 2;
  if (h->slopeflag != 0 || wetdry) {
    LimitArgs L{};
    L.m = h->mesh;
    L.ph = h->ph;
    L.q = h->q[irk].p;
    L.minmax = h->minmax.p;
    L.wd = h->wd.p;
    L.slopeflag = h->slopeflag;
    L.wetdry = wetdry ? 1 : 0;
    L.ne_act = h->n_own;
    L.err = h->err.p;
    if (h->slopeflag != 0) {
      LaunchTimer t(h, 1);
      h->v->node_minmax(L, grid_for(h->np, kPointBlock), h->stream);
      t.done();
    }
    LaunchTimer t(h, 2);
    h->v->limit_wetdry(L, h->limit_shape, h->stream);
    t.done();
  }
}

// Steps it0 .. it0+n-1: the host forcing of each chunk of steps is computed
// into pinned memory and copied with one transfer ahead of its kernels.
// MET_FORCING of NWS = 1 from the attached fort.22 (met_forcing.F:49-66):
// the next NP records, in the device node order, copied to the nodal fields
// the next stage kernel reads (stream-ordered after the previous stage's
// kernels); the stage kernel applies RAMPDG.
void met_stage(dgswem_cuda* h) {
  const int np = h->np, ng = h->np_glob;
  const int b = h->met_next;
  DG_CUDA(cudaEventSynchronize(h->met_done[b]));  // pinned block b free again
  h->met_in.resize(3 * (size_t)ng);
  double* in = h->met_in.data();
  met_read_block(h->met, in, in + ng, in + 2 * (size_t)ng);
  double* o = h->met_pin[b];
  for (int i = 0; i < np; ++i) {
    const int n = h->node_perm_h[i];
    o[i] = in[n];
    o[(size_t)np + i] = in[(size_t)ng + n];
    o[(size_t)2 * np + i] = in[(size_t)2 * ng + n];
  }
  const size_t bytes = (size_t)np * sizeof(double);
  DG_CUDA(cudaMemcpyAsync(h->wsx.p, o, bytes, cudaMemcpyHostToDevice, h->stream));
  DG_CUDA(cudaMemcpyAsync(h->wsy.p, o + np, bytes, cudaMemcpyHostToDevice, h->stream));
  DG_CUDA(cudaMemcpyAsync(h->pr.p, o + 2 * (size_t)np, bytes, cudaMemcpyHostToDevice, h->stream));
  DG_CUDA(cudaEventRecord(h->met_done[b], h->stream));
  h->met_next = b ^ 1;
}

void launch_stage(dgswem_cuda* h, int it, int irk, const double* forcing) {
  if (h->keep_wd)
    DG_CUDA(cudaMemcpyAsync(h->keep_wd[irk - 1], h->wd.p, (size_t)h->ne * sizeof(int), cudaMemcpyDeviceToDevice,
                            h->stream));
  launch_stage_rhs(h, it, irk, forcing);
  if (h->keep_pre)
    DG_CUDA(cudaMemcpyAsync(h->keep_pre[irk - 1], h->q[irk].p, 9 * (size_t)h->ne * sizeof(double),
                            cudaMemcpyDeviceToDevice, h->stream));
  launch_limit(h, irk);
}

// ---- CUDA graphs of whole steps ----
// A graph holds graph_steps (even) steps: one host-to-device copy of the
// chunk's stage blocks (the host forcing of the stage, then RAMPDG) and the
// stage kernels, which read the ramp and forcing from that block.  An even
// step count brings the swapped stage buffers back to the captured
// arrangement.
size_t graph_block(const dgswem_cuda* h) { return h->forcing_per_stage + 1; }

void graph_release(dgswem_cuda* h) {
  for (int b = 0; b < 2; ++b) {
    if (h->gexec[b]) cudaGraphExecDestroy(h->gexec[b]);
    if (h->graph[b]) cudaGraphDestroy(h->graph[b]);
    h->gexec[b] = nullptr;
    h->graph[b] = nullptr;
  }
  h->graph_ready = false;
}

void graph_fill(dgswem_cuda* h, double* buf, int it0) {
  const int nrk = h->nrk;
  const size_t blk = graph_block(h);
  for (int i = 0; i < h->graph_steps; ++i)
    for (int irk = 1; irk <= nrk; ++irk) {
      double timedg, rampdg;
      stage_clock(h, it0 + i, irk, &timedg, &rampdg);
      double* o = buf + ((size_t)i * nrk + (irk - 1)) * blk;
      if (h->forcing_per_stage) stage_forcing(h, timedg, rampdg, o);
      o[h->forcing_per_stage] = rampdg;
    }
}

void graph_capture(dgswem_cuda* h) {
  graph_release(h);
  const int m = h->graph_steps, nrk = h->nrk;
  const size_t blk = graph_block(h), len = (size_t)m * nrk * blk, bytes = len * sizeof(double);
  h->gbuf_dev.ensure(len);
  for (int b = 0; b < 2; ++b) {
    if (h->gdone[b]) DG_CUDA(cudaEventSynchronize(h->gdone[b]));
    if (h->gbuf_bytes < bytes && h->gbuf_host[b]) {
      cudaFreeHost(h->gbuf_host[b]);
      h->gbuf_host[b] = nullptr;
    }
    if (!h->gbuf_host[b]) DG_CUDA(cudaMallocHost(&h->gbuf_host[b], bytes));
    if (!h->gdone[b]) DG_CUDA(cudaEventCreateWithFlags(&h->gdone[b], cudaEventDisableTiming));
  }
  h->gbuf_bytes = std::max(h->gbuf_bytes, bytes);
  const long long l0 = h->launches;
  h->graph_q0 = h->q[0].p;
  for (int b = 0; b < 2; ++b) {
    DG_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed));
    try {
      DG_CUDA(cudaMemcpyAsync(h->gbuf_dev.p, h->gbuf_host[b], bytes, cudaMemcpyHostToDevice, h->stream));
      for (int i = 0; i < m; ++i) {
        for (int irk = 1; irk <= nrk; ++irk) {
          const double* sb = h->gbuf_dev.p + ((size_t)i * nrk + (irk - 1)) * blk;
          launch_stage_rhs(h, 0, irk, h->forcing_per_stage ? sb : nullptr, sb + h->forcing_per_stage);
          launch_limit(h, irk);
        }
        std::swap(h->q[0], h->q[nrk]);
      }
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(h->stream, &g);
      if (g) cudaGraphDestroy(g);
      h->launches = l0;
      throw;
    }
    DG_CUDA(cudaStreamEndCapture(h->stream, &h->graph[b]));
    DG_CUDA(cudaGraphInstantiate(&h->gexec[b], h->graph[b], 0));
  }
  h->graph_launches = (h->launches - l0) / 2;
  h->launches = l0;
  h->graph_ready = true;
}

// Steps it0 .. it0+n-1 through the graphs, as many whole graphs as fit;
// returns the steps done.
int run_steps_graph(dgswem_cuda* h, int it0, int n) {
  const int m = h->graph_steps, nrk = h->nrk;
  if (m < 2 || h->prof_on || n < m || h->met) return 0;
  if (!h->graph_ready) graph_capture(h);
  if (h->q[0].p != h->graph_q0) {  // the state sits in the other buffer: move it where the graphs read it
    DG_CUDA(cudaMemcpyAsync(h->q[nrk].p, h->q[0].p, 3 * (size_t)h->dofh * h->ne * sizeof(double),
                            cudaMemcpyDeviceToDevice, h->stream));
    std::swap(h->q[0], h->q[nrk]);
  }
  int done = 0, b = h->graph_next;
  for (; done + m <= n; done += m, b ^= 1) {
    DG_CUDA(cudaEventSynchronize(h->gdone[b]));  // buffer b free again
    graph_fill(h, h->gbuf_host[b], it0 + done);
    DG_CUDA(cudaGraphLaunch(h->gexec[b], h->stream));
    DG_CUDA(cudaEventRecord(h->gdone[b], h->stream));
    h->launches += h->graph_launches;
  }
  h->graph_next = b;
  return done;
}

void run_steps(dgswem_cuda* h, int it0, int n) {
  const int nrk = h->nrk;
  const int by_graph = run_steps_graph(h, it0, n);
  it0 += by_graph;
  n -= by_graph;
  for (int done = 0; done < n;) {
    const int m = std::min(n - done, h->chunk_steps > 0 ? h->chunk_steps : n);
    const double* dev = nullptr;
    if (h->forcing_per_stage) {
      if (h->forcing_copied) DG_CUDA(cudaEventSynchronize(h->forcing_copied));  // pinned buffer free again
      for (int i = 0; i < m; ++i)
        for (int irk = 1; irk <= nrk; ++irk) {
          double timedg, rampdg;
          stage_clock(h, it0 + done + i, irk, &timedg, &rampdg);
          stage_forcing(h, timedg, rampdg, h->forcing_host + ((size_t)i * nrk + (irk - 1)) * h->forcing_per_stage);
        }
      const size_t bytes = (size_t)m * nrk * h->forcing_per_stage * sizeof(double);
      DG_CUDA(cudaMemcpyAsync(h->forcing_dev.p, h->forcing_host, bytes, cudaMemcpyHostToDevice, h->stream));
      DG_CUDA(cudaEventRecord(h->forcing_copied, h->stream));
      dev = h->forcing_dev.p;
    }
    for (int i = 0; i < m; ++i) {
      const int it = it0 + done + i;
      for (int irk = 1; irk <= nrk; ++irk) {
        if (h->met) met_stage(h);
        launch_stage(h, it, irk, dev ? dev + ((size_t)i * nrk + (irk - 1)) * h->forcing_per_stage : nullptr);
      }
      std::swap(h->q[0], h->q[nrk]);  // stage NRK+1 becomes stage 1
    }
    done += m;
  }
}

// Nodal scratch of dgswem_cuda_modal2nodal_noalloc: ETA2, UU2, VV2 for up to
// kScratchNodes nodes, each array starting at a multiple of kScratchNodes.
// The CUDA loader reserves it with this module on each device; no call
// allocates it.
constexpr size_t kScratchNodes = DGSWEM_CUDA_NOALLOC_MAX_NODES;
static __device__ __align__(256) double g_nodal_scratch[3 * kScratchNodes];

// Device address of g_nodal_scratch on `device` (the current device), looked
// up once per device ordinal under a lock; fixed-size table, no allocation.
// Kept for the life of the process (the primary context is assumed not to be
// reset between calls).
constexpr int kMaxScratchDevices = 64;
std::mutex g_scratch_lock;
double* g_scratch_addr[kMaxScratchDevices] = {};

double* nodal_scratch(int device) {
  if (device < 0 || device >= kMaxScratchDevices)
    throw Failure(DGSWEM_ERR_ARG, "modal2nodal_noalloc: device ordinal " + std::to_string(device) +
                                      " outside [0, " + std::to_string(kMaxScratchDevices) + ")");
  std::lock_guard<std::mutex> guard(g_scratch_lock);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    DG_CUDA(cudaGetSymbolAddress(&p, g_nodal_scratch));
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  return g_scratch_addr[device];
}

}  // namespace

namespace {

// The scope of the discrete adjoint (adjoint.cu); DGSWEM_ERR_ARG otherwise.
// Allocates its buffers and zeroes the state cotangent and the gradients.
void adjoint_prepare(dgswem_cuda* h) {
  auto no = [](const char* what) {
    throw Failure(DGSWEM_ERR_ARG, std::string("the discrete adjoint does not cover ") + what);
  };
  if (h->nparts != 1) no("partitioned handles");
  if (h->v == &kMixed) no("the mixed-precision form (FP64 handles only)");
  if (!(h->ph.nleq == 1.0 && h->ph.leq == 0.0)) no("NLEQ=0 (linearised) runs");
  if (h->ph.ics != 1) no("ICS=2");
  if (h->nfeds > 0 || h->nreds > 0 || h->mesh.nebseg > 0 || h->mesh.nibseg > 0)
    no("flow, radiation or barrier boundaries");
  if (h->ph.iflinbf == 0 && h->ph.ifhybf == 1) no("hybrid friction");
  if (h->met) no("a fort.22 met file (give the fields with dgswem_cuda_set_met)");
  const size_t n9 = 9 * (size_t)h->ne;
  if (h->adj_lam.size() != (size_t)h->nrk + 1) {
    h->adj_lam.clear();
    h->adj_nu.clear();
    h->adj_lam.resize(h->nrk + 1);
    h->adj_nu.resize(h->nrk);
    for (auto& b : h->adj_lam) b.alloc(n9);
    for (auto& b : h->adj_nu) b.alloc(n9);
    h->adj_gn.alloc((size_t)h->ne);
    h->adj_ghb.alloc(3 * (size_t)h->ne);
    h->adj_eb.alloc(36 * (size_t)h->ne);
    if (h->slopeflag != 0 || h->nolifa >= 2) {
      h->adj_mm.alloc(6 * (size_t)h->np);
      h->adj_nb.alloc(6 * (size_t)h->np);
      h->adj_arg.alloc(6 * (size_t)h->np);
      h->adj_lb.alloc(18 * (size_t)h->ne);
      h->adj_pre_step.resize(h->nrk);
      for (auto& b : h->adj_pre_step) b.alloc(n9);
    }
    h->adj_wd_step.resize(h->nrk);
    for (auto& b : h->adj_wd_step) b.alloc((size_t)h->ne);
    // slots of edges in no list are never written: zero once
    DG_CUDA(cudaMemset(h->adj_eb.p, 0, 36 * (size_t)h->ne * sizeof(double)));
    std::vector<unsigned> info(h->ne);
    DG_CUDA(cudaMemcpy(info.data(), h->einfo.p, h->ne * sizeof(unsigned), cudaMemcpyDeviceToHost));
    std::vector<int> edges;
    for (int e = 0; e < h->ne; ++e)
      for (int l = 0; l < 3; ++l) {
        const unsigned k = ei_kind(info[e], l);
        if ((k == kInterior && ei_flag(info[e], l)) || k == kLand || k == kOcean) {
          edges.push_back(e);
          edges.push_back(l);
        }
      }
    h->adj_nedge = (int)(edges.size() / 2);
    h->adj_edges.upload(edges.empty() ? std::vector<int>(2, 0) : edges);
  }
  DG_CUDA(cudaMemsetAsync(h->adj_lam[h->nrk].p, 0, n9 * sizeof(double), h->stream));
  DG_CUDA(cudaMemsetAsync(h->adj_gn.p, 0, (size_t)h->ne * sizeof(double), h->stream));
  DG_CUDA(cudaMemsetAsync(h->adj_ghb.p, 0, 3 * (size_t)h->ne * sizeof(double), h->stream));
  h->adj_on = true;
}

// Carry the state cotangent adj_lam[nrk] back through step `it`, whose stage
// I state is stage[I-1], stage forcing `forcing` (nrk blocks of
// forcing_per_stage, or null) and, with the limiter, stage kernel outputs
// before the limiter pre[irk-1]; adds the step's parameter gradient.
void adjoint_stages(dgswem_cuda* h, int it, const double* const* stage, const double* forcing,
                    const double* const* pre, const int* const* wdst) {
  const bool limits = h->slopeflag != 0 || h->nolifa >= 2;
  const int nrk = h->nrk;
  const size_t n9 = 9 * (size_t)h->ne;
  // the pass of j = nrk+1 assigns every lam_I / nu_I, I <= nrk (no zeroing)
  for (int j = nrk + 1; j >= 1; --j) {
    if (j <= nrk) {
      AdjArgs a{};
      a.m = h->mesh;
      a.ph = h->ph;
      a.q = stage[j - 1];
      a.nu = h->adj_nu[j - 1].p;
      a.lam = h->adj_lam[j - 1].p;
      a.g_n = h->mesh.manning ? h->adj_gn.p : nullptr;
      a.g_hb = h->adj_ghb.p;
      a.ocean_zg = forcing ? forcing + (size_t)(j - 1) * h->forcing_per_stage : nullptr;
      a.pr = h->nws ? h->pr.p : nullptr;
      a.eb = h->adj_eb.p;
      a.edges = h->adj_edges.p;
      a.nedge = h->adj_nedge;
      a.wd = wdst[j - 1];
      double timedg;
      stage_clock(h, it, j, &timedg, &a.rampdg);
      adj::launch_rhs_vjp(a, h->stream);
      check_launch(h, "edge_vjp");
      check_launch(h, "elem_vjp");
    }
    if (j >= 2) {
      const int irk = j - 1;
      if (limits) {  // stage state j is the limited / wet-dried output of stage irk's kernel
        adj::launch_limit_vjp(h->mesh, h->ph, h->slopeflag, h->nolifa >= 2 ? 1 : 0, wdst[irk - 1], pre[irk - 1],
                              h->adj_mm.p, h->adj_arg.p, h->adj_lam[j - 1].p, h->adj_lb.p, h->adj_nb.p,
                              h->adj_ghb.p, h->stream);
        for (int k = 0; k < (h->slopeflag != 0 ? 4 : 1); ++k) check_launch(h, "limit_vjp");
      }
      SspAdjArgs b{};
      b.lam_j = h->adj_lam[j - 1].p;
      b.n = irk;
      b.first = j == nrk + 1;
      b.len = (long long)n9;
      for (int I = 1; I <= irk; ++I) {
        b.lam[I - 1] = h->adj_lam[I - 1].p;
        b.nu[I - 1] = h->adj_nu[I - 1].p;
        b.a[I - 1] = h->atvd[(size_t)(irk - 1) * nrk + (I - 1)];
        b.b[I - 1] = h->btvd[(size_t)(irk - 1) * nrk + (I - 1)] * h->dtdp;
      }
      adj::launch_ssp_adj(b, h->stream);
      check_launch(h, "ssp_adj");
    }
  }
  std::swap(h->adj_lam[0].p, h->adj_lam[nrk].p);  // the cotangent of stage 1 = of the step's start
}

void ensure_slot(dgswem_cuda* h, int slot) {
  if ((size_t)slot >= h->slot_q.size()) {
    h->slot_q.resize(slot + 1);
    h->slot_wd.resize(slot + 1);
  }
  if (!h->slot_q[slot].p) {
    h->slot_q[slot].alloc(9 * (size_t)h->ne);
    h->slot_wd[slot].alloc((size_t)h->ne);
  }
}

void save_slot(dgswem_cuda* h, int slot) {
  ensure_slot(h, slot);
  DG_CUDA(cudaMemcpyAsync(h->slot_q[slot].p, h->q[0].p, 9 * (size_t)h->ne * sizeof(double),
                          cudaMemcpyDeviceToDevice, h->stream));
  DG_CUDA(cudaMemcpyAsync(h->slot_wd[slot].p, h->wd.p, (size_t)h->ne * sizeof(int), cudaMemcpyDeviceToDevice,
                          h->stream));
}

void load_slot(dgswem_cuda* h, int slot) {
  if (slot < 0 || (size_t)slot >= h->slot_q.size() || !h->slot_q[slot].p)
    throw Failure(DGSWEM_ERR_ARG, "state slot " + std::to_string(slot) + " was never saved");
  DG_CUDA(cudaMemcpyAsync(h->q[0].p, h->slot_q[slot].p, 9 * (size_t)h->ne * sizeof(double),
                          cudaMemcpyDeviceToDevice, h->stream));
  DG_CUDA(cudaMemcpyAsync(h->wd.p, h->slot_wd[slot].p, (size_t)h->ne * sizeof(int), cudaMemcpyDeviceToDevice,
                          h->stream));
}

void seed_gauges(dgswem_cuda* h, const double* w_dev) {
  adj::launch_gauge_seed(h->adj_lam[h->nrk].p, h->ne, h->group_elem.p, h->group_ptr.p, h->group_gauge.p,
                         h->gauge_phi.p, w_dev, h->ngroup, h->stream);
  if (h->ngroup > 0) check_launch(h, "gauge_seed");
}

}  // namespace

extern "C" {

int dgswem_cuda_last_error(char* buf, int buflen) {
  if (!buf || buflen <= 0) return DGSWEM_ERR_ARG;
  std::strncpy(buf, g_last_error.c_str(), (size_t)buflen - 1);
  buf[buflen - 1] = 0;
  return DGSWEM_OK;
}

static dgswem_cuda* create_handle(const dgswem_cuda_setup* s, int part, int nparts, int device, int flags) {
  {
    if (flags & ~(DGSWEM_CUDA_STRICT | DGSWEM_CUDA_MIXED | DGSWEM_CUDA_FAST))
      throw Failure(DGSWEM_ERR_ARG, "unknown flags");
    if (((flags & DGSWEM_CUDA_STRICT) != 0) + ((flags & DGSWEM_CUDA_MIXED) != 0) + ((flags & DGSWEM_CUDA_FAST) != 0) > 1)
      throw Failure(DGSWEM_ERR_ARG, "DGSWEM_CUDA_STRICT, DGSWEM_CUDA_FAST and DGSWEM_CUDA_MIXED exclude each other");
    if (s->dofh != 3 && s->dofh != kP2Modes)
      throw Failure(DGSWEM_ERR_ARG, "DOFH must be 3 (p=1) or 6 (p=2)");
    if (s->dofh == kP2Modes) {
      if (nparts != 1) throw Failure(DGSWEM_ERR_ARG, "p=2 runs on a whole-mesh handle (dgswem_cuda_create)");
      if (s->slopeflag != 0) throw Failure(DGSWEM_ERR_ARG, "the slope limiter is p=1 only, as in the reference");
      if (s->nolifa >= 2) throw Failure(DGSWEM_ERR_ARG, "wetting and drying are p=1 only, as in the reference");
      if (s->ics != 1) throw Failure(DGSWEM_ERR_ARG, "p=2 supports ICS=1");
      if (s->nfeds || s->nreds || s->nebseg || s->nibseg)
        throw Failure(DGSWEM_ERR_ARG, "p=2 supports land and ocean boundaries (no flow, radiation or barriers)");
    }
    if (s->ne <= 0 || s->np <= 0 || s->nedges <= 0) throw Failure(DGSWEM_ERR_ARG, "empty mesh");
    if (s->nrk < 1 || s->nrk > kMaxStages) throw Failure(DGSWEM_ERR_ARG, "nrk out of range");
    if (s->nws != 0 && s->nws != 1) throw Failure(DGSWEM_ERR_ARG, "only NWS=0/1 are supported");
    if (s->nramp == 3) throw Failure(DGSWEM_ERR_ARG, "NRAMP = 3 not supported");
    if (s->ics != 1 && s->ics != 2) throw Failure(DGSWEM_ERR_ARG, "ICS must be 1 or 2");
    validate_mesh_ids(s);
    int ndev = 0;
    DG_CUDA(cudaGetDeviceCount(&ndev));
    (void)cudaGetLastError();  // drop an error left by other code on this thread
    if (device < 0 || device >= ndev) throw Failure(DGSWEM_ERR_ARG, "no such CUDA device");
    DG_CUDA(cudaSetDevice(device));
    std::unique_ptr<dgswem_cuda> h(new dgswem_cuda());
    h->device = device;
    // the strict kernels unless the fast or the mixed form is asked for
    h->v = (flags & DGSWEM_CUDA_FAST) ? &kFast : (flags & DGSWEM_CUDA_MIXED) ? &kMixed : &kStrict;
    h->dofh = s->dofh;
    if (h->dofh == kP2Modes) {
      h->v2 = (flags & DGSWEM_CUDA_FAST) ? &kFastP2 : (flags & DGSWEM_CUDA_MIXED) ? &kMixedP2 : &kStrictP2;
      h->tile_shape = kP2PlanShape;
    }
    h->ne = s->ne;
    h->np = s->np;
    h->nrk = s->nrk;
    h->nramp = s->nramp;
    h->slopeflag = s->slopeflag;
    h->nreds = s->nreds;
    h->nolifa = s->nolifa;
    h->nws = s->nws;
    h->dtdp = s->dtdp;
    h->statim = s->statim;
    h->dramp = s->dramp;
    h->atvd.assign(s->atvd, s->atvd + (size_t)s->nrk * s->nrk);
    h->btvd.assign(s->btvd, s->btvd + (size_t)s->nrk * s->nrk);
    h->dtvd.assign(s->dtvd, s->dtvd + s->nrk);
    h->keep_rhs.assign(s->nrk, 0);
    for (int I = 1; I <= s->nrk; ++I)
      for (int irk = I + 1; irk <= s->nrk; ++irk)
        if (h->btvd[(size_t)(irk - 1) * s->nrk + (I - 1)] != 0.0) h->keep_rhs[I - 1] = 1;
    Physics& p = h->ph;
    p.g = s->g;
    p.h0 = s->h0;
    p.dtdp = s->dtdp;
    p.nleq = s->nleq;
    p.leq = s->leq;
    p.nleqg = s->nleq * s->g;
    p.fg_l = s->leq * s->g;
    p.tau_cap = .9 * (1.0 / s->dtdp);
    p.cf = s->cf;
    p.hbreak = s->hbreak;
    p.ftheta = s->ftheta;
    p.fgamma = s->fgamma;
    p.iflinbf = s->iflinbf;
    p.ifhybf = s->ifhybf;
    p.ifnlfa = s->ifnlfa;
    p.nws = s->nws;
    p.rainfall = s->rainfall;
    p.ics = s->ics;
    DG_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    {
      const BasisP1 B = make_basis_p1();
      kFast.set_basis(B);
      kStrict.set_basis(B);
      kMixed.set_basis(B);
      adj::set_basis(B);
      if (h->v2) h->v2->set_basis(make_basis_p2());
      DG_CUDA(cudaGetLastError());
    }
    const PartPlan plan = make_part_plan(s, part, nparts);
    build_layout(h.get(), s, plan);
    build_halo(h.get(), s, plan);
    if (h->v2) {
      std::vector<unsigned> info(h->ne);
      DG_CUDA(cudaMemcpy(info.data(), h->einfo.p, h->ne * sizeof(unsigned), cudaMemcpyDeviceToHost));
      std::vector<int> edges;
      for (int e = 0; e < h->ne; ++e)
        for (int l = 0; l < 3; ++l) {
          const unsigned k = ei_kind(info[e], l);
          if ((k == kInterior && ei_flag(info[e], l)) || k == kLand || k == kOcean) {
            edges.push_back(e);
            edges.push_back(l);
          }
        }
      h->p2_nedge = (int)edges.size() / 2;
      h->p2_edges.upload(edges.empty() ? std::vector<int>(2, 0) : edges);
      int dev_smem = 0;
      DG_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
      const char* pair = std::getenv("DGSWEM_CUDA_P2_PAIR");
      h->p2_tiled = h->ntile > 0 && !(pair && std::atoi(pair) != 0) &&
                    h->v2->tile_smem(h->mesh.max_halo, std::max(h->mesh.max_tasks, 1)) <= (size_t)dev_smem;
      if (!h->p2_tiled) {  // the edge + element pair's flux slots (slots of edges in no list stay zero)
        h->p2_ef.alloc((size_t)3 * kP2Egp * 3 * h->ne);
        DG_CUDA(cudaMemset(h->p2_ef.p, 0, h->p2_ef.n * sizeof(double)));
      }
    }
    const size_t nl = (size_t)h->ne, npl = (size_t)h->np;
    h->q.resize(s->nrk + 1);
    for (auto& b : h->q) {
      b.alloc(3 * (size_t)h->dofh * nl);
      DG_CUDA(cudaMemset(b.p, 0, b.n * sizeof(double)));
    }
    h->rhs.resize(s->nrk);
    for (int I = 0; I < s->nrk; ++I)
      if (h->keep_rhs[I]) h->rhs[I].alloc(3 * (size_t)h->dofh * nl);
    h->wd.alloc(nl);
    h->wd_staging.alloc(s->ne);
    h->nodecode.alloc(s->np);
    h->minmax.alloc(6 * (size_t)npl);
    h->err.alloc(1);
    DG_CUDA(cudaMemset(h->err.p, 0, sizeof(unsigned)));
    if (s->nws == 1) {
      h->wsx.alloc(npl); h->wsy.alloc(npl); h->pr.alloc(npl);
      DG_CUDA(cudaMemset(h->wsx.p, 0, npl * sizeof(double)));
      DG_CUDA(cudaMemset(h->wsy.p, 0, npl * sizeof(double)));
      DG_CUDA(cudaMemset(h->pr.p, 0, npl * sizeof(double)));
    }
    // host-side boundary forcing (ocean and flow harmonics)
    h->needs = s->needs;
    h->nfeds = s->nfeds;
    if (!h->amig.empty()) {
      h->emo_h.assign(s->emo_dg, s->emo_dg + (size_t)s->nbfr * s->needs * 2);
      h->efa_h.assign(s->efa_dg, s->efa_dg + (size_t)s->nbfr * s->needs * 2);
    }
    if (!h->famig.empty()) {
      h->qnam_h.assign(s->qnam_dg, s->qnam_dg + (size_t)s->nffr * s->nfeds * 2);
      h->qnph_h.assign(s->qnph_dg, s->qnph_dg + (size_t)s->nffr * s->nfeds * 2);
    }
    h->forcing_per_stage = h->amig.size() * (size_t)s->needs * 2 + h->famig.size() * (size_t)s->nfeds * 3;
    if (h->forcing_per_stage) {
      const size_t per_step = h->forcing_per_stage * (size_t)s->nrk;
      h->chunk_steps = (int)std::max<size_t>(1, std::min<size_t>(512, (size_t)(8u << 20) / (per_step * sizeof(double))));
      DG_CUDA(cudaMallocHost(&h->forcing_host, per_step * h->chunk_steps * sizeof(double)));
      h->forcing_dev.alloc(per_step * h->chunk_steps);
      DG_CUDA(cudaEventCreateWithFlags(&h->forcing_copied, cudaEventDisableTiming));
    }
    upload_state(h.get(), s->ze, s->qx, s->qy, s->wdflg);
    return h.release();
  }
}

int dgswem_cuda_create(const dgswem_cuda_setup* s, int device, int flags, dgswem_cuda** out) {
  return guarded([&]() {
    if (!s || !out) throw Failure(DGSWEM_ERR_ARG, "null argument");
    *out = nullptr;
    *out = create_handle(s, 0, 1, device, flags);
  });
}

int dgswem_cuda_create_part(const dgswem_cuda_setup* s, int part, int nparts, int device, int flags,
                            dgswem_cuda** out) {
  return guarded([&]() {
    if (!s || !out) throw Failure(DGSWEM_ERR_ARG, "null argument");
    *out = nullptr;
    if (nparts < 1 || part < 0 || part >= nparts) throw Failure(DGSWEM_ERR_ARG, "partition index out of range");
    *out = create_handle(s, part, nparts, device, flags);
  });
}

void dgswem_cuda_destroy(dgswem_cuda* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& p : h->pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
  for (auto e : h->ev_pool) cudaEventDestroy(e);
  if (h->forcing_copied) cudaEventDestroy(h->forcing_copied);
  if (h->forcing_host) cudaFreeHost(h->forcing_host);
  if (h->met) dgswem_met_reader_close(h->met);
  for (int b = 0; b < 2; ++b) {
    if (h->met_done[b]) cudaEventDestroy(h->met_done[b]);
    if (h->met_pin[b]) cudaFreeHost(h->met_pin[b]);
  }
  graph_release(h);
  for (int b = 0; b < 2; ++b) {
    if (h->gdone[b]) cudaEventDestroy(h->gdone[b]);
    if (h->gbuf_host[b]) cudaFreeHost(h->gbuf_host[b]);
  }
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
}

int dgswem_cuda_hydro_timestep(dgswem_cuda* h, int it) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1)
      throw Failure(DGSWEM_ERR_ARG, "a partitioned handle steps through dgswem_cuda_stage_rhs / _stage_limit / "
                                    "_step_end with halo exchanges in between");
    DG_CUDA(cudaSetDevice(h->device));
    run_steps(h, it, 1);
  });
}

int dgswem_cuda_run(dgswem_cuda* h, int it0, int nsteps) {
  return guarded([&]() {
    if (!h || nsteps < 0) throw Failure(DGSWEM_ERR_ARG, "bad arguments");
    if (h->nparts != 1)
      throw Failure(DGSWEM_ERR_ARG, "a partitioned handle steps through dgswem_cuda_stage_rhs / _stage_limit / "
                                    "_step_end with halo exchanges in between");
    DG_CUDA(cudaSetDevice(h->device));
    run_steps(h, it0, nsteps);
  });
}

int dgswem_cuda_synchronize(dgswem_cuda* h) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    DG_CUDA(cudaStreamSynchronize(h->stream));
    unsigned e = 0;
    DG_CUDA(cudaMemcpy(&e, h->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (e) throw Failure(DGSWEM_ERR_NUMERIC, "NaN in the state produced on the device");
  });
}

int dgswem_cuda_upload_state(dgswem_cuda* h, const double* ze, const double* qx, const double* qy,
                             const int* wdflg) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    upload_state(h, ze, qx, qy, wdflg);
  });
}

int dgswem_cuda_download_state(dgswem_cuda* h, double* ze, double* qx, double* qy, int* wdflg) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    double* dst[3] = {ze, qx, qy};
    if (h->nparts == 1) {  // every element is owned: scatter to input order on the device
      const int ne = h->ne;
      const size_t dofh = (size_t)h->dofh;
      h->staging.ensure(3 * dofh * ne);
      for (int var = 0; var < 3; ++var) {
        if (!dst[var]) continue;
        double* sv = h->staging.p + dofh * ne * var;
        if (h->v2)
          h->v2->layout(false, h->q[0].p, sv, ne, var, h->inv.p, h->stream);
        else
          h->v->s2f(h->q[0].p, sv, ne, var, h->inv.p, grid_for(ne, kPointBlock), h->stream);
        check_launch(h, "soa_to_fortran");
        DG_CUDA(cudaMemcpyAsync(dst[var], sv, dofh * ne * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      }
      if (wdflg) {
        h->v->gather_int(h->wd.p, h->wd_staging.p, h->inv.p, ne, grid_for(ne, kPointBlock), h->stream);
        check_launch(h, "gather_int");
        DG_CUDA(cudaMemcpyAsync(wdflg, h->wd_staging.p, (size_t)ne * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      }
      DG_CUDA(cudaStreamSynchronize(h->stream));
      return;
    }
    // a partition: the owned elements' entries of the input-order arrays;
    // the others are left as they are
    const int no = h->n_own, nl = h->ne;
    std::vector<double> buf(3 * (size_t)no);
    std::vector<int> wbuf(no);
    for (int var = 0; var < 3; ++var) {
      if (!dst[var]) continue;
      for (int k = 0; k < 3; ++k)
        DG_CUDA(cudaMemcpyAsync(buf.data() + (size_t)k * no, h->q[0].p + (size_t)(3 * var + k) * nl,
                                (size_t)no * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      DG_CUDA(cudaStreamSynchronize(h->stream));
      for (int i = 0; i < no; ++i)
        for (int k = 0; k < 3; ++k) dst[var][(size_t)3 * h->perm_h[i] + k] = buf[(size_t)k * no + i];
    }
    if (wdflg) {
      DG_CUDA(cudaMemcpyAsync(wbuf.data(), h->wd.p, (size_t)no * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
      DG_CUDA(cudaStreamSynchronize(h->stream));
      for (int i = 0; i < no; ++i) wdflg[h->perm_h[i]] = wbuf[i];
    }
  });
}

int dgswem_cuda_met_file(dgswem_cuda* h, const char* path) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nws != 1) throw Failure(DGSWEM_ERR_ARG, "a fort.22 met file needs NWS = 1");
    need_p1(h, "dgswem_cuda_met_file");
    DG_CUDA(cudaSetDevice(h->device));
    if (h->met) {
      dgswem_met_reader_close(h->met);
      h->met = nullptr;
    }
    if (!path) return;
    dgswem_met_reader* r = nullptr;
    const int rc = dgswem_met_reader_open(path, h->np_glob, &r);
    if (rc != DGSWEM_OK) throw Failure(rc, std::string("fort.22: cannot open ") + path);
    h->met = r;
    for (int b = 0; b < 2; ++b) {
      if (!h->met_pin[b]) DG_CUDA(cudaMallocHost(&h->met_pin[b], 3 * (size_t)h->np * sizeof(double)));
      if (!h->met_done[b]) {
        DG_CUDA(cudaEventCreateWithFlags(&h->met_done[b], cudaEventDisableTiming));
        DG_CUDA(cudaEventRecord(h->met_done[b], h->stream));
      }
    }
  });
}

int dgswem_cuda_set_met(dgswem_cuda* h, const double* wsx2, const double* wsy2, const double* pr2) {
  return guarded([&]() {
    if (!h || !wsx2 || !wsy2 || !pr2) throw Failure(DGSWEM_ERR_ARG, "null argument");
    if (h->nws != 1) throw Failure(DGSWEM_ERR_ARG, "met forcing needs NWS = 1");
    DG_CUDA(cudaSetDevice(h->device));
    // the fields in the device node order
    const int np = h->np;
    std::vector<double> buf(3 * (size_t)np);
    for (int i = 0; i < np; ++i) {
      const int n = h->node_perm_h[i];
      buf[i] = wsx2[n];
      buf[(size_t)np + i] = wsy2[n];
      buf[(size_t)2 * np + i] = pr2[n];
    }
    const size_t bytes = (size_t)np * sizeof(double);
    DG_CUDA(cudaMemcpyAsync(h->wsx.p, buf.data(), bytes, cudaMemcpyHostToDevice, h->stream));
    DG_CUDA(cudaMemcpyAsync(h->wsy.p, buf.data() + np, bytes, cudaMemcpyHostToDevice, h->stream));
    DG_CUDA(cudaMemcpyAsync(h->pr.p, buf.data() + 2 * (size_t)np, bytes, cudaMemcpyHostToDevice, h->stream));
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_modal2nodal(dgswem_cuda* h, double* eta2, double* uu2, double* vv2, int* nodecode) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "modal2nodal needs the whole mesh (a handle of dgswem_cuda_create)");
    DG_CUDA(cudaSetDevice(h->device));
    const int np = h->np;
    h->staging.ensure(4 * (size_t)np);
    double* d = h->staging.p;
    if (h->v2)
      h->v2->modal2nodal(h->mesh, h->q[0].p, h->ph.nleq, h->ph.leq, d, d + np, d + 2 * (size_t)np, h->nodecode.p,
                         h->stream);
    else
      h->v->modal2nodal(h->mesh, h->q[0].p, h->wd.p, h->ph.nleq, h->ph.leq, d, d + np, d + 2 * (size_t)np,
                        h->nodecode.p, grid_for(np, kPointBlock), h->stream);
    check_launch(h, "modal2nodal");
    if (eta2) DG_CUDA(cudaMemcpyAsync(eta2, d, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (uu2) DG_CUDA(cudaMemcpyAsync(uu2, d + np, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (vv2) DG_CUDA(cudaMemcpyAsync(vv2, d + 2 * (size_t)np, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (nodecode)
      DG_CUDA(cudaMemcpyAsync(nodecode, h->nodecode.p, np * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_modal2nodal_noalloc(dgswem_cuda* h, double* eta2, double* uu2, double* vv2, int* nodecode) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_modal2nodal_noalloc");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "modal2nodal needs the whole mesh (a handle of dgswem_cuda_create)");
    const int np = h->np;
    if (np > DGSWEM_CUDA_NOALLOC_MAX_NODES)
      throw Failure(DGSWEM_ERR_ARG, "modal2nodal_noalloc: NP = " + std::to_string(np) +
                                        " exceeds the static scratch maximum DGSWEM_CUDA_NOALLOC_MAX_NODES = " +
                                        std::to_string(DGSWEM_CUDA_NOALLOC_MAX_NODES));
    DG_CUDA(cudaSetDevice(h->device));
    double* eta = nodal_scratch(h->device);
    double* uu = eta + kScratchNodes;
    double* vv = uu + kScratchNodes;
    h->v->modal2nodal(h->mesh, h->q[0].p, h->wd.p, h->ph.nleq, h->ph.leq, eta, uu, vv, h->nodecode.p,
                      grid_for(np, kPointBlock), h->stream);
    check_launch(h, "modal2nodal");
    if (eta2) DG_CUDA(cudaMemcpyAsync(eta2, eta, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (uu2) DG_CUDA(cudaMemcpyAsync(uu2, uu, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (vv2) DG_CUDA(cudaMemcpyAsync(vv2, vv, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (nodecode)
      DG_CUDA(cudaMemcpyAsync(nodecode, h->nodecode.p, np * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_stage_rhs(dgswem_cuda* h, int it, int irk) { return dgswem_cuda_stage_rhs_tiles(h, it, irk, 0); }

int dgswem_cuda_stage_rhs_tiles(dgswem_cuda* h, int it, int irk, int tiles) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_stage_rhs");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (irk < 1 || irk > h->nrk) throw Failure(DGSWEM_ERR_ARG, "stage out of range");
    if (tiles < 0 || tiles > 2) throw Failure(DGSWEM_ERR_ARG, "tiles must be 0 (all), 1 (interior) or 2 (boundary)");
    DG_CUDA(cudaSetDevice(h->device));
    if (tiles == kBoundaryTiles) {  // the stage's forcing was uploaded by its interior launch
      launch_stage_rhs(h, it, irk, h->forcing_per_stage ? h->forcing_dev.p : nullptr, nullptr, kBoundaryTiles);
      return;
    }
    const double* dev = nullptr;
    if (h->forcing_per_stage) {  // this stage's boundary forcing, host cos, one small copy
      if (h->forcing_copied) DG_CUDA(cudaEventSynchronize(h->forcing_copied));
      double timedg, rampdg;
      stage_clock(h, it, irk, &timedg, &rampdg);
      stage_forcing(h, timedg, rampdg, h->forcing_host);
      DG_CUDA(cudaMemcpyAsync(h->forcing_dev.p, h->forcing_host, h->forcing_per_stage * sizeof(double),
                              cudaMemcpyHostToDevice, h->stream));
      DG_CUDA(cudaEventRecord(h->forcing_copied, h->stream));
      dev = h->forcing_dev.p;
    }
    if (h->met) met_stage(h);
    launch_stage_rhs(h, it, irk, dev, nullptr, (TileSet)tiles);
  });
}

int dgswem_cuda_tile_split(const dgswem_cuda* h, int* n_interior, int* n_boundary) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    need_p1(h, "dgswem_cuda_tile_split");
    if (n_interior) *n_interior = h->n_tile_interior;
    if (n_boundary) *n_boundary = h->ntile - h->n_tile_interior;
  });
}

int dgswem_cuda_stage_limit(dgswem_cuda* h, int irk) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_stage_limit");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (irk < 1 || irk > h->nrk) throw Failure(DGSWEM_ERR_ARG, "stage out of range");
    DG_CUDA(cudaSetDevice(h->device));
    launch_limit(h, irk);
  });
}

int dgswem_cuda_step_end(dgswem_cuda* h) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_step_end");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    std::swap(h->q[0], h->q[h->nrk]);  // stage NRK+1 becomes stage 1
  });
}

int dgswem_cuda_part_info(const dgswem_cuda* h, int* part, int* nparts, int* n_owned, int* n_local) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (part) *part = h->part;
    if (nparts) *nparts = h->nparts;
    if (n_owned) *n_owned = h->n_own;
    if (n_local) *n_local = h->ne;
  });
}

int dgswem_cuda_halo_count(const dgswem_cuda* h, int kind, int peer, int* nsend, int* nrecv) {
  return guarded([&]() {
    if (!h || !nsend || !nrecv) throw Failure(DGSWEM_ERR_ARG, "null argument");
    if (kind != kHaloMeans && kind != kHaloFull) throw Failure(DGSWEM_ERR_ARG, "unknown halo kind");
    if (peer < 0 || peer >= h->nparts) throw Failure(DGSWEM_ERR_ARG, "peer out of range");
    *nsend = (int)(h->halo_off[kind][0][peer + 1] - h->halo_off[kind][0][peer]);
    *nrecv = (int)(h->halo_off[kind][1][peer + 1] - h->halo_off[kind][1][peer]);
  });
}

static int halo_copy(dgswem_cuda* h, int kind, int peer, int irk, double* buf, bool pack) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_halo_pack / _unpack");
    if (!h || !buf) throw Failure(DGSWEM_ERR_ARG, "null argument");
    if (kind != kHaloMeans && kind != kHaloFull) throw Failure(DGSWEM_ERR_ARG, "unknown halo kind");
    if (peer < 0 || peer >= h->nparts) throw Failure(DGSWEM_ERR_ARG, "peer out of range");
    if (irk < 0 || irk > h->nrk) throw Failure(DGSWEM_ERR_ARG, "stage buffer out of range");
    DG_CUDA(cudaSetDevice(h->device));
    const auto& off = h->halo_off[kind][pack ? 0 : 1];
    const int n = (int)(off[peer + 1] - off[peer]);
    h->v->halo(pack, h->q[irk].p, h->wd.p, h->ne, h->halo_idx.p + off[peer], n, kind, buf, h->stream);
    if (n > 0) check_launch(h, pack ? "halo_pack" : "halo_unpack");
  });
}

int dgswem_cuda_halo_pack(dgswem_cuda* h, int kind, int peer, int irk, double* buf) {
  return halo_copy(h, kind, peer, irk, buf, true);
}

int dgswem_cuda_halo_unpack(dgswem_cuda* h, int kind, int peer, int irk, const double* buf) {
  return halo_copy(h, kind, peer, irk, const_cast<double*>(buf), false);
}

long long dgswem_cuda_kernel_launches(const dgswem_cuda* h) { return h ? h->launches : -1; }

int dgswem_cuda_set_graph(dgswem_cuda* h, int steps) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (steps != 0 && (steps < 2 || steps % 2 != 0))
      throw Failure(DGSWEM_ERR_ARG, "steps per graph must be 0 (off) or an even number >= 2");
    DG_CUDA(cudaSetDevice(h->device));
    DG_CUDA(cudaStreamSynchronize(h->stream));
    graph_release(h);
    h->graph_steps = steps;
    h->graph_next = 0;
  });
}

namespace {

// Rebuilds the stage tile plan for tile shape `shape` from the device copies
// of the edge graph (link, einfo); on failure (the shape's plan does not fit
// the task word or shared memory) the current plan stays.  Captured graphs
// hold the old plan's launches: released.
void replan(dgswem_cuda* h, int shape) {
  DG_CUDA(cudaStreamSynchronize(h->stream));
  graph_release(h);
  std::vector<int> link(3 * (size_t)h->ne);
  std::vector<unsigned> info(h->ne);
  DG_CUDA(cudaMemcpy(link.data(), h->link.p, link.size() * sizeof(int), cudaMemcpyDeviceToHost));
  DG_CUDA(cudaMemcpy(info.data(), h->einfo.p, info.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
  const int old = h->tile_shape;
  h->tile_shape = shape;
  try {
    build_tile_plan(h, h->n_own, h->ne, link, info);
  } catch (...) {
    h->tile_shape = old;  // the plan is uploaded only after every check passed
    throw;
  }
}

// Mesh signature of the autotuner's cache: the variant, the device, the
// element / node counts and a hash of the edge graph (FNV-1a over einfo and
// link) and of the physics switches that decide which kernels run.
uint64_t tune_signature(dgswem_cuda* h) {
  std::vector<int> link(3 * (size_t)h->ne);
  std::vector<unsigned> info(h->ne);
  DG_CUDA(cudaMemcpy(link.data(), h->link.p, link.size() * sizeof(int), cudaMemcpyDeviceToHost));
  DG_CUDA(cudaMemcpy(info.data(), h->einfo.p, info.size() * sizeof(unsigned), cudaMemcpyDeviceToHost));
  uint64_t x = 1469598103934665603ull;
  auto mix = [&](uint64_t v) {
    for (int b = 0; b < 8; ++b) {
      x ^= (v >> (8 * b)) & 0xffu;
      x *= 1099511628211ull;
    }
  };
  mix((uint64_t)(uintptr_t)h->v);
  mix((uint64_t)h->device);
  mix((uint64_t)h->ne);
  mix((uint64_t)h->np);
  mix((uint64_t)h->nrk);
  mix((uint64_t)h->slopeflag);
  mix((uint64_t)h->nolifa);
  mix((uint64_t)(h->ph.nleq == 1.0 && h->ph.leq == 0.0));
  mix((uint64_t)(h->mesh.sfac_edge != nullptr));
  for (unsigned v : info) mix(v);
  for (int v : link) mix((uint64_t)(unsigned)v);
  return x;
}

struct TuneResult {
  int tile_shape, limit_shape;
  double ms_tile[kNumTileShapes], ms_limit[kNumLimitShapes];
};
std::mutex g_tune_lock;
std::map<uint64_t, TuneResult> g_tune_cache;

}  // namespace

static_assert(kNumTileShapes <= DGSWEM_CUDA_MAX_SHAPES && kNumLimitShapes <= DGSWEM_CUDA_MAX_SHAPES,
              "shape lists fit the C-ABI arrays");

int dgswem_cuda_shapes(int* n_tile, int* tile_elems, int* tile_threads, int* n_limit, int* limit_threads,
                       int* limit_blocks_per_sm) {
  return guarded([&]() {
    if (n_tile) *n_tile = kNumTileShapes;
    if (n_limit) *n_limit = kNumLimitShapes;
    for (int i = 0; i < kNumTileShapes; ++i) {
      if (tile_elems) tile_elems[i] = kTileShapes[i].tile;
      if (tile_threads) tile_threads[i] = kTileShapes[i].threads;
    }
    for (int i = 0; i < kNumLimitShapes; ++i) {
      if (limit_threads) limit_threads[i] = kLimitBlocks[i];
      if (limit_blocks_per_sm) limit_blocks_per_sm[i] = kLimitMinBlocks[i];
    }
  });
}

int dgswem_cuda_set_shapes(dgswem_cuda* h, int tile_shape, int limit_shape) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_set_shapes");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (tile_shape < -1 || tile_shape >= kNumTileShapes || limit_shape < -1 || limit_shape >= kNumLimitShapes)
      throw Failure(DGSWEM_ERR_ARG, "shape index out of range");
    DG_CUDA(cudaSetDevice(h->device));
    if (tile_shape >= 0 && tile_shape != h->tile_shape) replan(h, tile_shape);
    if (limit_shape >= 0) h->limit_shape = limit_shape;
  });
}

int dgswem_cuda_get_shapes(const dgswem_cuda* h, int* tile_shape, int* limit_shape) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (tile_shape) *tile_shape = (h->dofh == 6 && !h->p2_tiled) ? -1 : h->tile_shape;
    if (limit_shape) *limit_shape = h->limit_shape;
  });
}

int dgswem_cuda_autotune(dgswem_cuda* h, int it, int steps, int reps, int flags, double* ms_tile,
                         double* ms_limit) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_autotune");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (steps < 1 || reps < 1 || it < 1) throw Failure(DGSWEM_ERR_ARG, "autotune: it, steps and reps must be >= 1");
    if (h->nparts != 1)
      throw Failure(DGSWEM_ERR_ARG, "autotune times whole steps of a handle of dgswem_cuda_create");
    DG_CUDA(cudaSetDevice(h->device));
    DG_CUDA(cudaStreamSynchronize(h->stream));
    const uint64_t sig = tune_signature(h);
    TuneResult r{};
    bool cached = false;
    if (flags & DGSWEM_CUDA_TUNE_CACHED) {
      std::lock_guard<std::mutex> g(g_tune_lock);
      auto f = g_tune_cache.find(sig);
      if (f != g_tune_cache.end()) {
        r = f->second;
        cached = true;
      }
    }
    if (!cached) {
      // the state the steps start from: kept, restored before each timing
      // and at the end (the stage buffers other than q[0] and the limiter's
      // node bounds are scratch of every step)
      const size_t n9 = 9 * (size_t)h->ne;
      DevBuf<double> q0;
      DevBuf<int> wd0;
      DevBuf<unsigned> err0;
      q0.alloc(n9);
      wd0.alloc((size_t)h->ne);
      err0.alloc(1);
      DG_CUDA(cudaMemcpyAsync(q0.p, h->q[0].p, n9 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
      DG_CUDA(cudaMemcpyAsync(wd0.p, h->wd.p, (size_t)h->ne * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
      DG_CUDA(cudaMemcpyAsync(err0.p, h->err.p, sizeof(unsigned), cudaMemcpyDeviceToDevice, h->stream));
      auto restore = [&]() {
        DG_CUDA(cudaMemcpyAsync(h->q[0].p, q0.p, n9 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        DG_CUDA(cudaMemcpyAsync(h->wd.p, wd0.p, (size_t)h->ne * sizeof(int), cudaMemcpyDeviceToDevice, h->stream));
        DG_CUDA(cudaMemcpyAsync(h->err.p, err0.p, sizeof(unsigned), cudaMemcpyDeviceToDevice, h->stream));
      };
      const int graph_steps = h->graph_steps;
      const bool prof_on = h->prof_on;
      const int tile0 = h->tile_shape, limit0 = h->limit_shape;
      h->graph_steps = 0;
      h->prof_on = false;
      cudaEvent_t ev[2] = {nullptr, nullptr};
      auto time_steps = [&]() -> double {
        restore();
        run_steps(h, it, 1);  // warm-up (first launch of the shape's kernels)
        double best = 0.0;
        for (int k = 0; k < reps; ++k) {
          restore();
          DG_CUDA(cudaEventRecord(ev[0], h->stream));
          run_steps(h, it, steps);
          DG_CUDA(cudaEventRecord(ev[1], h->stream));
          DG_CUDA(cudaEventSynchronize(ev[1]));
          float ms = 0.f;
          DG_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
          const double per = (double)ms / steps;
          if (k == 0 || per < best) best = per;
        }
        return best;
      };
      try {
        for (auto& e : ev) DG_CUDA(cudaEventCreate(&e));
        r.tile_shape = -1;
        for (int s = 0; s < kNumTileShapes; ++s) {
          r.ms_tile[s] = -1.0;
          try {
            replan(h, s);
          } catch (const Failure& f) {
            if (f.code != DGSWEM_ERR_ARG) throw;
            continue;  // the shape's plan does not fit: not timed
          }
          r.ms_tile[s] = time_steps();
          if (r.tile_shape < 0 || r.ms_tile[s] < r.ms_tile[r.tile_shape]) r.tile_shape = s;
        }
        if (r.tile_shape < 0) throw Failure(DGSWEM_ERR_ARG, "autotune: no tile shape fits the mesh");
        if (h->tile_shape != r.tile_shape) replan(h, r.tile_shape);
        const bool limiter = h->slopeflag != 0 || h->nolifa >= 2;
        r.limit_shape = limit0;
        for (int s = 0; s < kNumLimitShapes; ++s) r.ms_limit[s] = -1.0;
        if (limiter) {
          for (int s = 0; s < kNumLimitShapes; ++s) {
            h->limit_shape = s;
            r.ms_limit[s] = time_steps();
            if (s == 0 || r.ms_limit[s] < r.ms_limit[r.limit_shape]) r.limit_shape = s;
          }
        }
        restore();
      } catch (...) {
        for (auto& e : ev)
          if (e) cudaEventDestroy(e);
        h->graph_steps = graph_steps;
        h->prof_on = prof_on;
        try {
          restore();
          h->limit_shape = limit0;
          if (h->tile_shape != tile0) replan(h, tile0);
        } catch (...) {
        }
        throw;
      }
      for (auto& e : ev) cudaEventDestroy(e);
      h->graph_steps = graph_steps;
      h->prof_on = prof_on;
      DG_CUDA(cudaStreamSynchronize(h->stream));
      std::lock_guard<std::mutex> g(g_tune_lock);
      g_tune_cache[sig] = r;
    }
    if (h->tile_shape != r.tile_shape) replan(h, r.tile_shape);
    h->limit_shape = r.limit_shape;
    if (ms_tile)
      for (int s = 0; s < kNumTileShapes; ++s) ms_tile[s] = r.ms_tile[s];
    if (ms_limit)
      for (int s = 0; s < kNumLimitShapes; ++s) ms_limit[s] = r.ms_limit[s];
  });
}

int dgswem_cuda_set_stream(dgswem_cuda* h, void* stream) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    prof_flush(h);
    DG_CUDA(cudaStreamSynchronize(h->stream));
    h->stream = static_cast<cudaStream_t>(stream);
  });
}

void* dgswem_cuda_stream(const dgswem_cuda* h) { return h ? static_cast<void*>(h->stream) : nullptr; }

int dgswem_cuda_profile(dgswem_cuda* h, int enable) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    prof_flush(h);
    for (int k = 0; k < 4; ++k) { h->prof_ms[k] = 0.0; h->prof_n[k] = 0; }
    h->prof_on = enable != 0;
  });
}

int dgswem_cuda_profile_read(dgswem_cuda* h, double* ms, long long* launches) {
  return guarded([&]() {
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    prof_flush(h);
    for (int k = 0; k < 4; ++k) {
      if (ms) ms[k] = h->prof_ms[k];
      if (launches) launches[k] = h->prof_n[k];
    }
  });
}


// ---- parameters, state slots, gauges and the discrete adjoint ---------------
// (no counterparts in the reference)

int dgswem_cuda_set_params(dgswem_cuda* h, const double* nbar, const double* hb) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_set_params");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "set_params needs the whole mesh (a handle of dgswem_cuda_create)");
    DG_CUDA(cudaSetDevice(h->device));
    DG_CUDA(cudaStreamSynchronize(h->stream));
    const int ne = h->ne;
    if (nbar) {
      if (!h->mesh.manning) throw Failure(DGSWEM_ERR_ARG, "set_params: the deck has no Manning n (NWP / fort.13)");
      std::vector<double> row(ne);
      for (int i = 0; i < ne; ++i) row[i] = nbar[h->perm_h[i]];
      DG_CUDA(cudaMemcpy(h->egeo.p + (size_t)EGeo::kNbar * ne, row.data(), ne * sizeof(double),
                         cudaMemcpyHostToDevice));
      if (h->egeof.p) {
        std::vector<float> rf(row.begin(), row.end());
        DG_CUDA(cudaMemcpy(h->egeof.p + (size_t)EGeo::kNbar * ne, rf.data(), ne * sizeof(float),
                           cudaMemcpyHostToDevice));
      }
    }
    if (hb) {
      std::vector<double> d(3 * (size_t)ne);
      for (int k = 0; k < 3; ++k)
        for (int i = 0; i < ne; ++i) d[(size_t)k * ne + i] = hb[3 * (size_t)h->perm_h[i] + k];
      DG_CUDA(cudaMemcpy(h->hb.p, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
  });
}

int dgswem_cuda_state_save(dgswem_cuda* h, int slot) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_state_save");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (slot < 0) throw Failure(DGSWEM_ERR_ARG, "negative state slot");
    DG_CUDA(cudaSetDevice(h->device));
    save_slot(h, slot);
  });
}

int dgswem_cuda_state_load(dgswem_cuda* h, int slot) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_state_load");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    load_slot(h, slot);
  });
}

int dgswem_cuda_gauges(dgswem_cuda* h, int ng, const int* elem, const double* phi) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_gauges");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "gauges need the whole mesh (a handle of dgswem_cuda_create)");
    if (ng < 0 || (ng > 0 && (!elem || !phi))) throw Failure(DGSWEM_ERR_ARG, "gauges: bad arguments");
    DG_CUDA(cudaSetDevice(h->device));
    std::vector<int> inv(h->ne);
    for (int i = 0; i < h->ne; ++i) inv[h->perm_h[i]] = i;
    std::vector<int> ed(std::max(ng, 1), 0);
    for (int g = 0; g < ng; ++g) {
      if (elem[g] < 1 || elem[g] > h->ne) throw Failure(DGSWEM_ERR_ARG, "gauge element outside 1..NE");
      ed[g] = inv[elem[g] - 1];
    }
    h->ngauge = ng;
    h->gauge_elem.upload(ed);
    h->gauge_phi.upload(ng > 0 ? std::vector<double>(phi, phi + 3 * (size_t)ng) : std::vector<double>(3, 0.0));
    h->gauge_val.alloc(std::max(ng, 1));
    // distinct elements, each with its gauges in input order
    std::vector<int> order(ng);
    for (int g = 0; g < ng; ++g) order[g] = g;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ed[a] < ed[b]; });
    std::vector<int> gel, gptr(1, 0), ggauge;
    for (int i = 0; i < ng; ++i) {
      if (i == 0 || ed[order[i]] != ed[order[i - 1]]) {
        if (i) gptr.push_back(i);
        gel.push_back(ed[order[i]]);
      }
      ggauge.push_back(order[i]);
    }
    gptr.push_back(ng);
    h->ngroup = (int)gel.size();
    h->group_elem.upload(gel.empty() ? std::vector<int>(1, 0) : gel);
    h->group_ptr.upload(gptr);
    h->group_gauge.upload(ggauge.empty() ? std::vector<int>(1, 0) : ggauge);
  });
}

int dgswem_cuda_gauge_eta(dgswem_cuda* h, double* eta) {
  return guarded([&]() {
    if (!h || !eta) throw Failure(DGSWEM_ERR_ARG, "null argument");
    DG_CUDA(cudaSetDevice(h->device));
    if (h->ngauge == 0) return;
    adj::launch_gauge_eval(h->q[0].p, h->ne, h->gauge_elem.p, h->gauge_phi.p, h->ngauge, h->gauge_val.p,
                           h->stream);
    check_launch(h, "gauge_eval");
    DG_CUDA(cudaMemcpyAsync(eta, h->gauge_val.p, h->ngauge * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_adjoint_begin(dgswem_cuda* h) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_adjoint_begin");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    DG_CUDA(cudaSetDevice(h->device));
    adjoint_prepare(h);
  });
}

int dgswem_cuda_adjoint_seed(dgswem_cuda* h, const double* w) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_adjoint_seed");
    if (!h || !w) throw Failure(DGSWEM_ERR_ARG, "null argument");
    if (!h->adj_on) throw Failure(DGSWEM_ERR_ARG, "call dgswem_cuda_adjoint_begin first");
    DG_CUDA(cudaSetDevice(h->device));
    if (h->ngauge == 0) return;
    // from pageable memory the copy has read w when it returns
    DG_CUDA(cudaMemcpyAsync(h->gauge_val.p, w, h->ngauge * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    seed_gauges(h, h->gauge_val.p);
  });
}

int dgswem_cuda_adjoint_step(dgswem_cuda* h, int it) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_adjoint_step");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (!h->adj_on) throw Failure(DGSWEM_ERR_ARG, "call dgswem_cuda_adjoint_begin first");
    DG_CUDA(cudaSetDevice(h->device));
    // recompute step `it` from the loaded state: stage I's state is q[I-1]
    // (I >= 2) and q[nrk] (I = 1, swapped there at the end of the step)
    const int nrk = h->nrk;
    const bool limits = h->slopeflag != 0 || h->nolifa >= 2;
    std::vector<double*> pre(nrk, nullptr);
    std::vector<int*> wdk(nrk, nullptr);
    for (int I = 0; I < nrk; ++I) {
      if (limits) pre[I] = h->adj_pre_step[I].p;
      wdk[I] = h->adj_wd_step[I].p;
    }
    h->keep_pre = limits ? pre.data() : nullptr;
    h->keep_wd = wdk.data();
    try {
      run_steps(h, it, 1);
    } catch (...) {
      h->keep_pre = nullptr;
      h->keep_wd = nullptr;
      throw;
    }
    h->keep_pre = nullptr;
    h->keep_wd = nullptr;
    std::vector<const double*> st(nrk), pc(pre.begin(), pre.end());
    std::vector<const int*> wc(wdk.begin(), wdk.end());
    for (int I = 1; I <= nrk; ++I) st[I - 1] = I == 1 ? h->q[nrk].p : h->q[I - 1].p;
    adjoint_stages(h, it, st.data(), h->forcing_per_stage ? h->forcing_dev.p : nullptr, pc.data(), wc.data());
  });
}

int dgswem_cuda_misfit_forward(dgswem_cuda* h, int it0, int nsteps, int every, double* eta) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_misfit_forward");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (nsteps < 0 || every < 1) throw Failure(DGSWEM_ERR_ARG, "misfit_forward: bad step counts");
    DG_CUDA(cudaSetDevice(h->device));
    const int ng = h->ngauge;
    h->eta_rec.ensure(std::max<size_t>((size_t)nsteps * ng, 1));
    for (int k = 0; k < nsteps; ++k) {
      if (k % every == 0) save_slot(h, k / every);
      run_steps(h, it0 + k, 1);
      if (ng > 0) {
        adj::launch_gauge_eval(h->q[0].p, h->ne, h->gauge_elem.p, h->gauge_phi.p, ng, h->eta_rec.p + (size_t)k * ng,
                               h->stream);
        check_launch(h, "gauge_eval");
      }
    }
    if (eta && ng > 0 && nsteps > 0)
      DG_CUDA(cudaMemcpyAsync(eta, h->eta_rec.p, (size_t)nsteps * ng * sizeof(double), cudaMemcpyDeviceToHost,
                              h->stream));
    DG_CUDA(cudaStreamSynchronize(h->stream));
    unsigned err = 0;
    DG_CUDA(cudaMemcpy(&err, h->err.p, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) throw Failure(DGSWEM_ERR_NUMERIC, "NaN in the state during misfit_forward");
  });
}

int dgswem_cuda_adjoint_sweep(dgswem_cuda* h, int it0, int nsteps, int every, const double* w) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_adjoint_sweep");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (nsteps < 1 || every < 1) throw Failure(DGSWEM_ERR_ARG, "adjoint_sweep: bad step counts");
    DG_CUDA(cudaSetDevice(h->device));
    adjoint_prepare(h);
    const int nrk = h->nrk, ng = h->ngauge;
    const int nseg = (nsteps + every - 1) / every;
    for (int s = 0; s < nseg; ++s)
      if ((size_t)s >= h->slot_q.size() || !h->slot_q[s].p)
        throw Failure(DGSWEM_ERR_ARG, "adjoint_sweep: run dgswem_cuda_misfit_forward with the same steps first");
    if (ng > 0) {
      h->w_rec.ensure((size_t)nsteps * ng);
      DG_CUDA(cudaMemcpyAsync(h->w_rec.p, w, (size_t)nsteps * ng * sizeof(double), cudaMemcpyHostToDevice,
                              h->stream));
    }
    const size_t n9 = 9 * (size_t)h->ne, fstep = (size_t)nrk * h->forcing_per_stage;
    const int seg_steps = std::min(every, nsteps);
    if (h->adj_stage.size() < (size_t)seg_steps * (nrk - 1)) {
      h->adj_stage.resize((size_t)seg_steps * (nrk - 1));
      for (auto& b : h->adj_stage)
        if (!b.p) b.alloc(n9);
    }
    if (fstep) h->adj_forc.ensure(fstep * seg_steps);
    const bool limits = h->slopeflag != 0 || h->nolifa >= 2;
    if (limits && h->adj_pre.size() < (size_t)seg_steps * nrk) {
      h->adj_pre.resize((size_t)seg_steps * nrk);
      for (auto& b : h->adj_pre)
        if (!b.p) b.alloc(n9);
    }
    if (h->adj_wd.size() < (size_t)seg_steps * nrk) {
      h->adj_wd.resize((size_t)seg_steps * nrk);
      for (auto& b : h->adj_wd)
        if (!b.p) b.alloc((size_t)h->ne);
    }
    std::vector<const double*> st(nrk), pc(nrk, nullptr);
    std::vector<const int*> wc(nrk, nullptr);
    std::vector<double*> keep(nrk, nullptr);
    std::vector<int*> keepw(nrk, nullptr);
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int k0 = seg * every, k1 = std::min(k0 + every, nsteps);
      // forward over the segment, keeping each step's start state, stage
      // states and stage forcing
      load_slot(h, seg);
      for (int k = k0; k < k1; ++k) {
        const int j = k - k0;
        save_slot(h, nseg + j);
        for (int I = 0; I < nrk; ++I) {
          if (limits) keep[I] = h->adj_pre[(size_t)j * nrk + I].p;
          keepw[I] = h->adj_wd[(size_t)j * nrk + I].p;
        }
        h->keep_pre = limits ? keep.data() : nullptr;
        h->keep_wd = keepw.data();
        try {
          run_steps(h, it0 + k, 1);
        } catch (...) {
          h->keep_pre = nullptr;
          h->keep_wd = nullptr;
          throw;
        }
        h->keep_pre = nullptr;
        h->keep_wd = nullptr;
        for (int I = 2; I <= nrk; ++I)
          DG_CUDA(cudaMemcpyAsync(h->adj_stage[(size_t)j * (nrk - 1) + (I - 2)].p, h->q[I - 1].p,
                                  n9 * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        if (fstep)
          DG_CUDA(cudaMemcpyAsync(h->adj_forc.p + (size_t)j * fstep, h->forcing_dev.p, fstep * sizeof(double),
                                  cudaMemcpyDeviceToDevice, h->stream));
      }
      // backward: step k maps state k-1 to state k
      for (int k = k1; k > k0; --k) {
        const int j = k - 1 - k0;
        if (ng > 0) seed_gauges(h, h->w_rec.p + (size_t)(k - 1) * ng);
        st[0] = h->slot_q[nseg + j].p;
        for (int I = 2; I <= nrk; ++I) st[I - 1] = h->adj_stage[(size_t)j * (nrk - 1) + (I - 2)].p;
        for (int I = 0; I < nrk; ++I) {
          if (limits) pc[I] = h->adj_pre[(size_t)j * nrk + I].p;
          wc[I] = h->adj_wd[(size_t)j * nrk + I].p;
        }
        adjoint_stages(h, it0 + k - 1, st.data(), fstep ? h->adj_forc.p + (size_t)j * fstep : nullptr, pc.data(),
                       wc.data());
      }
    }
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_adjoint_read(dgswem_cuda* h, double* g_nbar, double* g_hb, double* lam_ze, double* lam_qx,
                             double* lam_qy) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_adjoint_read");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (!h->adj_on) throw Failure(DGSWEM_ERR_ARG, "call dgswem_cuda_adjoint_begin first");
    DG_CUDA(cudaSetDevice(h->device));
    const int ne = h->ne;
    DG_CUDA(cudaStreamSynchronize(h->stream));
    std::vector<double> gn(ne), gh(3 * (size_t)ne), lam(9 * (size_t)ne);
    DG_CUDA(cudaMemcpy(gn.data(), h->adj_gn.p, ne * sizeof(double), cudaMemcpyDeviceToHost));
    DG_CUDA(cudaMemcpy(gh.data(), h->adj_ghb.p, gh.size() * sizeof(double), cudaMemcpyDeviceToHost));
    DG_CUDA(cudaMemcpy(lam.data(), h->adj_lam[h->nrk].p, lam.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (int i = 0; i < ne; ++i) {
      const size_t e = (size_t)h->perm_h[i];
      if (g_nbar) g_nbar[e] = h->mesh.manning ? gn[i] : 0.0;
      for (int k = 0; k < 3; ++k) {
        if (g_hb) g_hb[3 * e + k] = gh[(size_t)k * ne + i];
        if (lam_ze) lam_ze[3 * e + k] = lam[(size_t)k * ne + i];
        if (lam_qx) lam_qx[3 * e + k] = lam[(size_t)(3 + k) * ne + i];
        if (lam_qy) lam_qy[3 * e + k] = lam[(size_t)(6 + k) * ne + i];
      }
    }
  });
}

int dgswem_cuda_limit_state(dgswem_cuda* h) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_limit_state");
    if (!h) throw Failure(DGSWEM_ERR_ARG, "null handle");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "limit_state needs the whole mesh (a handle of dgswem_cuda_create)");
    DG_CUDA(cudaSetDevice(h->device));
    launch_limit(h, 0);  // the stage path's SLOPELIMITER5 (+ WETDRY) on the current state
    DG_CUDA(cudaStreamSynchronize(h->stream));
  });
}

int dgswem_cuda_limiter_vjp(dgswem_cuda* h, const double* lam_ze, const double* lam_qx, const double* lam_qy,
                            double* out_ze, double* out_qx, double* out_qy) {
  return guarded([&]() {
    need_p1(h, "dgswem_cuda_limiter_vjp");
    if (!h || !lam_ze || !lam_qx || !lam_qy || !out_ze || !out_qx || !out_qy)
      throw Failure(DGSWEM_ERR_ARG, "null argument");
    if (h->nparts != 1) throw Failure(DGSWEM_ERR_ARG, "limiter_vjp needs the whole mesh");
    if (h->slopeflag == 0 && h->nolifa < 2)
      throw Failure(DGSWEM_ERR_ARG, "the deck has neither the slope limiter nor WETDRY");
    DG_CUDA(cudaSetDevice(h->device));
    adjoint_prepare(h);
    const int ne = h->ne;
    const size_t n9 = 9 * (size_t)ne;
    std::vector<double> lam(n9);
    const double* src[3] = {lam_ze, lam_qx, lam_qy};
    for (int var = 0; var < 3; ++var)
      for (int i = 0; i < ne; ++i)
        for (int k = 0; k < 3; ++k) lam[(size_t)(3 * var + k) * ne + i] = src[var][3 * (size_t)h->perm_h[i] + k];
    DG_CUDA(cudaMemcpy(h->adj_lam[0].p, lam.data(), n9 * sizeof(double), cudaMemcpyHostToDevice));
    adj::launch_limit_vjp(h->mesh, h->ph, h->slopeflag, h->nolifa >= 2 ? 1 : 0, h->wd.p, h->q[0].p, h->adj_mm.p,
                          h->adj_arg.p, h->adj_lam[0].p, h->adj_lb.p, h->adj_nb.p, h->adj_ghb.p, h->stream);
    for (int k = 0; k < (h->slopeflag != 0 ? 4 : 1); ++k) check_launch(h, "limit_vjp");
    DG_CUDA(cudaStreamSynchronize(h->stream));
    DG_CUDA(cudaMemcpy(lam.data(), h->adj_lam[0].p, n9 * sizeof(double), cudaMemcpyDeviceToHost));
    double* dst[3] = {out_ze, out_qx, out_qy};
    for (int var = 0; var < 3; ++var)
      for (int i = 0; i < ne; ++i)
        for (int k = 0; k < 3; ++k) dst[var][3 * (size_t)h->perm_h[i] + k] = lam[(size_t)(3 * var + k) * ne + i];
  });
}

}  // extern "C"
