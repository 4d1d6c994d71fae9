// hydro_kernels.cuh -- sm_100a kernels of one RK stage of the p=1 DG hydro
// step.  Per stage: stage_p1 (tile kernel: edge fluxes once per edge in
// shared memory, volume integral, SSP combination; no atomics) ->
// node_minmax (slope limiter node pass) -> limit_wetdry (limiter element
// pass + WETDRY).  Every arithmetic sequence follows the reference routine
// named in its comment.  Compiled twice (kernels_fast.cu with FMA
// contraction, kernels_strict.cu without), see hydro_device.cuh.
#pragma once

#include <cuda_runtime.h>

#include "hydro_device.cuh"

#ifndef DGSWEM_VARIANT
#error "define DGSWEM_VARIANT (fast or strict) before including hydro_kernels.cuh"
#endif

namespace dgswem {
namespace DGSWEM_VARIANT {

__constant__ BasisP1 cBasis;

struct Flux3 {
  double f, g, h;
};

// numerical_flux.F:750-914, Local Lax-Friedrichs.  kNonlin specialises
// NLEQ=1, LEQ=0 (the products with 1 and sums with 0 it removes are exact).
template <bool kNonlin>
__device__ __forceinline__ Flux3 llf(const Physics& P, double ze_in, double ze_ex, double qx_in,
                                     double qx_ex, double qy_in, double qy_ex, double hb_in,
                                     double hb_ex, double sf_in, double sf_ex, double nx, double ny,
                                     double G) {
  const double NLEQ = kNonlin ? 1.0 : P.nleq;
  const double LEQ = kNonlin ? 0.0 : P.leq;
  const double nleqg = G * NLEQ;
  const double j1 = ze_ex - ze_in, j2 = qx_ex - qx_in, j3 = qy_ex - qy_in;
  double ht_in, f1, fx1i, fy1i, fh, ui, vi, fx2i, fy2i, fx3i, fy3i;
  {
    ht_in = kNonlin ? ze_in + hb_in : ze_in * NLEQ + hb_in;
    f1 = kNonlin ? 1.0 : NLEQ + LEQ * hb_in;
    fx1i = qx_in * f1 * sf_in;
    fy1i = qy_in * f1;
    const double fu = kNonlin ? qx_in : NLEQ * qx_in;
    const double fv = kNonlin ? qy_in : NLEQ * qy_in;
    const double fg = nleqg * ze_in;
    fh = 1.0 / (kNonlin ? ht_in : NLEQ * ht_in + LEQ);
    ui = qx_in * fh;
    vi = qy_in * fh;
    const double huu = fu * ui, hvv = fv * vi, huv = fu * vi;
    const double gh2 = kNonlin ? fg * (0.5 * ze_in + hb_in) : fg * (0.5 * ze_in + hb_in) + P.fg_l * ze_in;
    fx2i = (huu + gh2) * sf_in;
    fy2i = huv;
    fx3i = huv * sf_in;
    fy3i = hvv + gh2;
  }
  double ht_ex, fx1e, fy1e, ue, ve, fx2e, fy2e, fx3e, fy3e;
  {
    ht_ex = kNonlin ? ze_ex + hb_ex : ze_ex * NLEQ + hb_ex;
    const double f1e = kNonlin ? 1.0 : NLEQ + LEQ * hb_ex;
    fx1e = qx_ex * f1e * sf_ex;
    fy1e = qy_ex * f1e;
    const double fu = kNonlin ? qx_ex : NLEQ * qx_ex;
    const double fv = kNonlin ? qy_ex : NLEQ * qy_ex;
    const double fg = nleqg * ze_ex;
    const double fhe = 1.0 / (kNonlin ? ht_ex : NLEQ * ht_ex + LEQ);
    ue = qx_ex * fhe;
    ve = qy_ex * fhe;
    const double huu = fu * ue, hvv = fv * ve, huv = fu * ve;
    const double gh2 = kNonlin ? fg * (0.5 * ze_ex + hb_ex) : fg * (0.5 * ze_ex + hb_ex) + P.fg_l * ze_ex;
    fx2e = (huu + gh2) * sf_ex;
    fy2e = huv;
    fx3e = huv * sf_ex;
    fy3e = hvv + gh2;
  }
  const double f1a = 0.5 * ((fx1i + fx1e) * nx + (fy1i + fy1e) * ny);
  const double f2a = 0.5 * ((fx2i + fx2e) * nx + (fy2i + fy2e) * ny);
  const double f3a = 0.5 * ((fx3i + fx3e) * nx + (fy3i + fy3e) * ny);
  const double uni = kNonlin ? ui * nx + vi * ny : (ui * nx + vi * ny) * NLEQ;
  const double nxsi = nx * sf_in, nxse = nx * sf_ex;
  const double ci = sqrt(G * ht_in * (ny * ny + nxsi * nxsi));
  const double une = kNonlin ? ue * nx + ve * ny : (ue * nx + ve * ny) * NLEQ;
  const double ce = sqrt(G * ht_ex * (ny * ny + nxse * nxse));
  const double eig = fmax(fmax(fmax(fabs(uni + ci), fabs(uni)), fmax(fabs(uni - ci), fabs(une + ce))),
                          fmax(fabs(une), fabs(une - ce)));
  Flux3 r;
  r.f = f1a - 0.5 * eig * j1;
  if (kNonlin) {
    r.g = f2a - 0.5 * eig * j2;
    r.h = f3a - 0.5 * eig * j3;
  } else {
    const double nx2 = NLEQ + LEQ * nx * nx, ny2 = NLEQ + LEQ * ny * ny, nxy = nx * ny;
    r.g = f2a - 0.5 * eig * (j2 * nx2 + LEQ * j3 * nxy);
    r.h = f3a - 0.5 * eig * (j3 * ny2 + LEQ * j2 * nxy);
  }
  return r;
}

__device__ __forceinline__ void load_basis(BasisP1& s) {
  const double* src = reinterpret_cast<const double*>(&cBasis);
  double* dst = reinterpret_cast<double*>(&s);
  for (int i = threadIdx.x; i < (int)(sizeof(BasisP1) / sizeof(double)); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
}

// Trace of the modal state at point j of local edge l (mode 1 is 1 there).
__device__ __forceinline__ void edge_trace(const BasisP1& B, const double* q, int l, int j, double& z,
                                           double& u, double& v) {
  const double p1 = B.phi_edge[l][j][1], p2 = B.phi_edge[l][j][2];
  z = q[0] + q[1] * p1 + q[2] * p2;
  u = q[3] + q[4] * p1 + q[5] * p2;
  v = q[6] + q[7] * p1 + q[8] * p2;
}

// Exterior (ghost) state of a boundary edge point from the in-side trace
// (land_edge_hydro.F:201-218, ocean_edge_hydro.F:148-177 and 255-259,
// flow_edge_hydro.F:126-150, radiation_edge_hydro.F:173-193,
// ebarrier_edge_hydro.F:120-160).  Point j of the edge, normal (nx, ny).
__device__ __forceinline__ void ghost_state(const StageArgs& A, const BasisP1& B, unsigned kind, int list, int j,
                                            double zi, double xi, double yi, double hbi, double nx, double ny,
                                            double& zx, double& xx, double& yx) {
  const Physics& P = A.ph;
  const double tx = -ny, ty = nx;
  zx = zi;
  xx = xi;
  yx = yi;
  if (kind == kOcean) {
    // endpoint values EMO*RFF*COS(ARGJ-EFA) come from the host for this stage
    double zsum = 0.0;
    for (int f = 0; f < A.m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * A.m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * B.xegp[j]);
    }
    zx = zsum;
    if (zx * P.ifnlfa + hbi <= 0) zx = fabs(hbi) + P.h0;
  } else if (kind == kLand) {
    const double qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const double qne = -qn, qte = qt, den = 1.0 / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  } else if (kind == kFlow) {
    // per-point terms QNAM_GP*RFF*COS(ARG) come from the host for this stage
    double qne = 0.0;
    xx = 0.0;
    yx = 0.0;
    for (int f = 0; f < A.m.nffr; ++f) {
      qne = qne + A.flow_qn[((size_t)f * A.m.nfeds + list) * 3 + j];
      xx = -(ty * qne - ny * 0.0) / (nx * ty - ny * tx);
      yx = -(-tx * qne + nx * 0.0) / (nx * ty - ny * tx);
    }
  } else if (kind == kRadiation) {
    const double qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const double qne = -qn + 2 * sqrt(P.g / (hbi + zi)) * zi, qte = qt, den = 1.0 / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  } else if (kind == kEBarrier) {
    const double above = zi - A.m.ebht[list];
    const double subsup = 2.0 * above / 3.0;
    double qne, qte;
    if (above < 0.01) {
      qne = -(xi * nx + yi * ny);
      qte = xi * tx + yi * ty;
    } else {
      qne = A.rampdg * A.m.ebcfsp[list] * subsup * sqrt(subsup * P.g);
      qte = 0.0;
    }
    xx = (ty * qne - ny * qte) / (nx * ty - ny * tx);
    yx = (-tx * qne + nx * qte) / (nx * ty - ny * tx);
  }
}

__device__ __forceinline__ void edge_geometry(const double* xs, const double* ys, int l, double& xlen,
                                              double& nx, double& ny) {
  // calc_normal.F:41-48 on this element's counter-clockwise edge l
  const int a = (l + 1) % 3, b = (l + 2) % 3;
  const double dy = ys[b] - ys[a], dx = xs[b] - xs[a];
  xlen = sqrt(dy * dy + dx * dx);
  nx = (ys[b] - ys[a]) / xlen;
  ny = -(xs[b] - xs[a]) / xlen;
}

// ibarrier_edge_hydro.F:21-607 for one side of internal-barrier segment `seg`;
// both elements of a segment evaluate the whole weir logic and keep their
// own part, so no element writes another's right-hand side.
template <bool kNonlin>
__device__ __noinline__ void ibarrier_side(const StageArgs& A, int seg, int side, double* out9) {
  const BasisP1& B = cBasis;
  const Physics& P = A.ph;
  const MeshView& m = A.m;
  const int ne = m.ne;
  const int elb = m.ib_elem[2 * seg], elf = m.ib_elem[2 * seg + 1];
  const int ledb = m.ib_led[2 * seg], ledf = m.ib_led[2 * seg + 1];
  const int wdb = A.wd[elb], wdf = A.wd[elf];
  for (int c = 0; c < 9; ++c) out9[c] = 0.0;
  if (wdb == 0 && wdf == 0) return;
  double qb[9], qf[9], hbb[3], hbf[3], xb[3], yb[3], xf[3], yf[3];
  for (int c = 0; c < 9; ++c) { qb[c] = A.qin[(size_t)c * ne + elb]; qf[c] = A.qin[(size_t)c * ne + elf]; }
  for (int k = 0; k < 3; ++k) { hbb[k] = m.hb[(size_t)k * ne + elb]; hbf[k] = m.hb[(size_t)k * ne + elf]; }
  for (int v = 0; v < 3; ++v) {
    const int nb = m.nm[(size_t)v * ne + elb], nf = m.nm[(size_t)v * ne + elf];
    xb[v] = m.x[nb]; yb[v] = m.y[nb]; xf[v] = m.x[nf]; yf[v] = m.y[nf];
  }
  double lenb, nxb, nyb, lenf, nxf, nyf;
  edge_geometry(xb, yb, ledb, lenb, nxb, nyb);
  edge_geometry(xf, yf, ledf, lenf, nxf, nyf);
  const double txb = -nyb, tyb = nxb, txf = -nyf, tyf = nxf;
  const double areasb = (xb[0] - xb[2]) * (yb[1] - yb[2]) + (xb[2] - xb[1]) * (yb[0] - yb[2]);
  const double areasf = (xf[0] - xf[2]) * (yf[1] - yf[2]) + (xf[2] - xf[1]) * (yf[0] - yf[2]);
  for (int i = 0; i < 3; ++i) {
    const int gpb = i, gpf = 2 - i;
    double zeb, qxb, qyb, zef, qxf, qyf;
    edge_trace(B, qb, ledb, gpb, zeb, qxb, qyb);
    edge_trace(B, qf, ledf, gpf, zef, qxf, qyf);
    const double hbbp = hbb[0] + hbb[1] * B.phi_edge[ledb][gpb][1] + hbb[2] * B.phi_edge[ledb][gpb][2];
    const double hbfp = hbf[0] + hbf[1] * B.phi_edge[ledf][gpf][1] + hbf[2] * B.phi_edge[ledf][gpf][2];
    const double sfb = m.sfac_edge ? m.sfac_edge[(size_t)(ledb * 3 + gpb) * ne + elb] : 1.0;
    const double sff = m.sfac_edge ? m.sfac_edge[(size_t)(ledf * 3 + gpf) * ne + elf] : 1.0;
    double aboveb = 0.0, abovef = 0.0;
    if (wdb == 1) aboveb = zeb - m.ibht[seg];
    if (wdf == 1) abovef = zef - m.ibht[seg];
    double qbn = 0.0, qfn = 0.0, qbt = 0.0, qft = 0.0;
    int weir = 0;
    if ((abovef <= 0.01 && aboveb <= 0.01) || fabs(abovef - aboveb) < 0.01) {
      qbn = -(qxb * nxb + qyb * nyb);
      qfn = -(qxf * nxf + qyf * nyf);
      qbt = qxb * txb + qyb * tyb;
      qft = qxf * txf + qyf * tyf;
    } else {
      const double ssf = 2.0 * abovef / 3.0, ssb = 2.0 * aboveb / 3.0;
      if (abovef > aboveb && abovef > 0.01) {
        weir = 1;
        qfn = (aboveb > ssf) ? A.rampdg * m.ibcfsb[seg] * aboveb * sqrt(2.0 * P.g * (abovef - aboveb))
                             : A.rampdg * m.ibcfsp[seg] * ssf * sqrt(ssf * P.g);
      } else if (aboveb > abovef && aboveb > 0.01) {
        weir = -1;
        qbn = (abovef > ssb) ? A.rampdg * m.ibcfsb[seg] * abovef * sqrt(2.0 * P.g * (aboveb - abovef))
                             : A.rampdg * m.ibcfsp[seg] * ssb * sqrt(ssb * P.g);
      }
    }
    Flux3 fb{0, 0, 0}, ff{0, 0, 0};
    double qxe = 0.0, qye = 0.0;
    bool done = false;
    if (weir <= 0) {
      qxe = (tyb * qbn - nyb * qbt) / (nxb * tyb - nyb * txb);
      qye = (-txb * qbn + nxb * qbt) / (nxb * tyb - nyb * txb);
      fb = llf<kNonlin>(P, zeb, zeb, qxb, qxe, qyb, qye, hbbp, hbbp, sfb, sfb, nxb, nyb, P.g);
      if (weir < 0) {  // the front side keeps the back side's exterior momentum
        ff = llf<kNonlin>(P, zef, zef, qxf, qxe, qyf, qye, hbfp, hbfp, sff, sff, nxf, nyf, wdf == 0 ? 0.0 : P.g);
        done = true;
      }
    }
    if (!done && weir >= 0) {
      qxe = (tyf * qfn - nyf * qft) / (nxf * tyf - nyf * txf);
      qye = (-txf * qfn + nxf * qft) / (nxf * tyf - nyf * txf);
      ff = llf<kNonlin>(P, zef, zef, qxf, qxe, qyf, qye, hbfp, hbfp, sff, sff, nxf, nyf, P.g);
      if (weir > 0)
        fb = llf<kNonlin>(P, zeb, zeb, qxb, qxe, qyb, qye, hbbp, hbbp, sfb, sfb, nxb, nyb, wdb == 0 ? 0.0 : P.g);
    }
    const Flux3 fo = side == 0 ? fb : ff;
    const int led = side == 0 ? ledb : ledf, gp = side == 0 ? gpb : gpf;
    const double areas = side == 0 ? areasb : areasf, len = side == 0 ? lenb : lenf;
    for (int k = 0; k < 3; ++k) {
      const double w = 2.0 * B.m_inv[k] / areas * len * B.phi_edge[led][gp][k] * B.wegp[gp];
      out9[k] = out9[k] - w * fo.f;
      out9[3 + k] = out9[3 + k] - w * fo.g;
      out9[6 + k] = out9[6 + k] - w * fo.h;
    }
  }
}

// ---------------------------------------------------------------------------
// Tile stage kernel.  A block owns kStageBlock consecutive elements and runs
// three phases separated by barriers:
//   1. per element: modal state, bathymetry and geometry into shared memory;
//      a block-wide prefix sum turns the edges this tile evaluates (boundary
//      edges, edges to elements of other tiles, and shared interior edges
//      once, from the reference's "in" element NEDEL(1)) into a dense task list;
//   2. per (task, Lobatto point): one LLF evaluation in the reference's own
//      in/ex orientation with its dry-side rules -> F, G_in, H_in, G_ex, H_ex;
//   3. per element: edge contributions in the reference's order (boundary
//      edges, then interior edges in edge-number order, the slot sum of
//      add_internal_flux), rain, volume integral, SSP combination.
// internal_edge_hydro.F, *_edge_hydro.F, rhs_dg_hydro.F, DG_hydro_timestep.F:238-290
// ---------------------------------------------------------------------------

// resident stage blocks per SM the register allocation targets
#ifndef DGSWEM_STAGE_MIN_BLOCKS
#define DGSWEM_STAGE_MIN_BLOCKS 4
#endif

// task word layout (int4 .x); .y in-side element, .z ex-side element or list
struct TaskBits {
  static constexpr int kKind = 0;      // 3 bits
  static constexpr int kInLocal = 3;   // in-side element is in this tile
  static constexpr int kExLocal = 4;   // ex-side element is in this tile
  static constexpr int kLedIn = 5;     // 2 bits
  static constexpr int kLedEx = 7;     // 2 bits
  static constexpr int kFlip = 9;      // owner is the ex side: normal = -owner's normal
  static constexpr int kOwner = 10;    // 8 bits, owner's local index
  static constexpr int kOwnerLed = 18; // 2 bits
};

struct TileShared {
  BasisP1 B;
  double q[12][kStageBlock];    // ZE, QX, QY modes and HB modes
  double geo[14][kStageBlock];  // AREAS; per local edge XLEN, nx, ny; y3-y1, y1-y2, x1-x3, x2-x1
  int wd[kStageBlock];
  int task_of[3][kStageBlock];
  int warp_sum[kStageBlock / 32];
  int ntask;
};

// dynamic shared memory: TileShared, then the task list (int4 each), then
// 15 doubles of results per task
constexpr size_t kTaskOffset = (sizeof(TileShared) + 15) / 16 * 16;
__host__ __device__ constexpr size_t stage_shared_bytes(int max_tasks) {
  return kTaskOffset + (size_t)(max_tasks + 1) * (sizeof(int4) + 15 * sizeof(double));
}

// One point of a tile task: (modal state of a side, its local edge, point)
__device__ __forceinline__ void side_trace(const TileShared& S, const StageArgs& A, bool local, int el, int led,
                                           int gp, double& z, double& u, double& v, double& h) {
  const double p1 = S.B.phi_edge[led][gp][1], p2 = S.B.phi_edge[led][gp][2];
  const int ne = A.m.ne;
  if (local) {
    z = S.q[0][el] + S.q[1][el] * p1 + S.q[2][el] * p2;
    u = S.q[3][el] + S.q[4][el] * p1 + S.q[5][el] * p2;
    v = S.q[6][el] + S.q[7][el] * p1 + S.q[8][el] * p2;
    h = S.q[9][el] + S.q[10][el] * p1 + S.q[11][el] * p2;
  } else {
    const double* q = A.qin;
    z = q[el] + q[(size_t)ne + el] * p1 + q[(size_t)2 * ne + el] * p2;
    u = q[(size_t)3 * ne + el] + q[(size_t)4 * ne + el] * p1 + q[(size_t)5 * ne + el] * p2;
    v = q[(size_t)6 * ne + el] + q[(size_t)7 * ne + el] * p1 + q[(size_t)8 * ne + el] * p2;
    const double* hb = A.m.hb;
    h = hb[el] + hb[(size_t)ne + el] * p1 + hb[(size_t)2 * ne + el] * p2;
  }
}

template <bool kNonlin>
__global__ void __launch_bounds__(kStageBlock, DGSWEM_STAGE_MIN_BLOCKS) stage_p1(const __grid_constant__ StageArgs A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  TileShared& S = *reinterpret_cast<TileShared*>(smem_raw);
  int4* tasks = reinterpret_cast<int4*>(smem_raw + kTaskOffset);
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const int ne = m.ne;
  const int tid = threadIdx.x;
  const int tile0 = blockIdx.x * kStageBlock;
  const int e = tile0 + tid;
  const bool valid = e < ne;
  const int ntile = min(kStageBlock, ne - tile0);
  {
    const double* src = reinterpret_cast<const double*>(&cBasis);
    double* dst = reinterpret_cast<double*>(&S.B);
    for (int i = tid; i < (int)(sizeof(BasisP1) / sizeof(double)); i += blockDim.x) dst[i] = src[i];
  }

  // ---- phase 1: element data, ownership, dense task list ----
  unsigned info = 0u;
  int link[3] = {-1, -1, -1};
  int own[3] = {0, 0, 0};
  int nown = 0;
  if (valid) {
#pragma unroll
    for (int c = 0; c < 9; ++c) S.q[c][tid] = A.qin[(size_t)c * ne + e];
#pragma unroll
    for (int k = 0; k < 3; ++k) S.q[9 + k][tid] = m.hb[(size_t)k * ne + e];
    S.wd[tid] = A.wd[e];
    double xs[3], ys[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const int nd = m.nm[(size_t)v * ne + e];
      xs[v] = m.x[nd];
      ys[v] = m.y[nd];
    }
    // AREAS (read_input.F:1406); XLEN and normals (calc_normal.F:41-48) on
    // this element's counter-clockwise edges
    S.geo[0][tid] = (xs[0] - xs[2]) * (ys[1] - ys[2]) + (xs[2] - xs[1]) * (ys[0] - ys[2]);
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      const int a = (l + 1) % 3, b = (l + 2) % 3;
      const double dy = ys[b] - ys[a], dx = xs[b] - xs[a];
      const double len = sqrt(dy * dy + dx * dx);
      S.geo[1 + 3 * l][tid] = len;
      S.geo[2 + 3 * l][tid] = (ys[b] - ys[a]) / len;
      S.geo[3 + 3 * l][tid] = -(xs[b] - xs[a]) / len;
    }
    S.geo[10][tid] = ys[2] - ys[0];
    S.geo[11][tid] = ys[0] - ys[1];
    S.geo[12][tid] = xs[0] - xs[2];
    S.geo[13][tid] = xs[1] - xs[0];
    info = m.einfo[e];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      link[l] = m.link[(size_t)l * ne + e];
      const unsigned kind = ei_kind(info, l);
      if (kind == kNone || kind == kIBarrier) continue;
      if (kind == kInterior) {
        const bool nbr_local = link[l] >= tile0 && link[l] < tile0 + ntile;
        own[l] = (!nbr_local || ei_flag(info, l)) ? 1 : 0;
      } else {
        own[l] = 1;
      }
      nown += own[l];
    }
  }
  // block exclusive scan of the owned-task counts
  const int lane = tid & 31, warp = tid >> 5;
  int incl = nown;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += t;
  }
  if (lane == 31) S.warp_sum[warp] = incl;
  __syncthreads();
  int base = incl - nown;
  for (int w = 0; w < warp; ++w) base += S.warp_sum[w];
  if (tid == blockDim.x - 1) S.ntask = base + nown;
  if (valid) {
#pragma unroll
    for (int l = 0; l < 3; ++l) {
      S.task_of[l][tid] = -1;
      if (!own[l]) continue;
      const unsigned kind = ei_kind(info, l);
      int4 t;
      unsigned fl = kind;
      fl |= (unsigned)tid << TaskBits::kOwner;
      fl |= (unsigned)l << TaskBits::kOwnerLed;
      if (kind == kInterior) {
        const int nb = link[l];
        const bool nbr_local = nb >= tile0 && nb < tile0 + ntile;
        const unsigned nled = ei_nled(info, l);
        if (ei_flag(info, l)) {  // this element is NEDEL(1): the in side
          fl |= 1u << TaskBits::kInLocal;
          fl |= (unsigned)l << TaskBits::kLedIn;
          fl |= nled << TaskBits::kLedEx;
          if (nbr_local) fl |= 1u << TaskBits::kExLocal;
          t.y = tid;
          t.z = nbr_local ? nb - tile0 : nb;
        } else {                 // the neighbour (another tile) is the in side
          fl |= 1u << TaskBits::kExLocal;
          fl |= nled << TaskBits::kLedIn;
          fl |= (unsigned)l << TaskBits::kLedEx;
          fl |= 1u << TaskBits::kFlip;
          t.y = nb;
          t.z = tid;
        }
      } else {
        fl |= 1u << TaskBits::kInLocal;
        fl |= (unsigned)l << TaskBits::kLedIn;
        t.y = tid;
        t.z = link[l];
      }
      t.x = (int)fl;
      t.w = 0;
      S.task_of[l][tid] = base;
      tasks[base] = t;
      ++base;
    }
  }
  __syncthreads();
  if (valid) {  // shared interior edges: read the owner's task
#pragma unroll
    for (int l = 0; l < 3; ++l)
      if (ei_kind(info, l) == kInterior && !own[l])
        S.task_of[l][tid] = S.task_of[ei_nled(info, l)][link[l] - tile0];
  }

  // ---- phase 2: one LLF per (task, point) ----
  double* res = reinterpret_cast<double*>(tasks + S.ntask + (S.ntask & 1));  // [task][point][5]
  const int nwork = 3 * S.ntask;
  for (int w = tid; w < nwork; w += blockDim.x) {
    const int ti = w / 3, I = w - 3 * ti;
    const int4 t = tasks[ti];
    const unsigned fl = (unsigned)t.x;
    const unsigned kind = fl & 7u;
    const bool in_local = (fl >> TaskBits::kInLocal) & 1u, ex_local = (fl >> TaskBits::kExLocal) & 1u;
    const int led_in = (fl >> TaskBits::kLedIn) & 3, led_ex = (fl >> TaskBits::kLedEx) & 3;
    const int owner = (fl >> TaskBits::kOwner) & 255, oled = (fl >> TaskBits::kOwnerLed) & 3;
    double nx = S.geo[2 + 3 * oled][owner], ny = S.geo[3 + 3 * oled][owner];
    if ((fl >> TaskBits::kFlip) & 1u) { nx = -nx; ny = -ny; }
    const int wd_in = in_local ? S.wd[t.y] : A.wd[t.y];
    const int gin = in_local ? tile0 + t.y : t.y;  // global ids for the ics=2 tables
    double* out = res + ((size_t)ti * 3 + I) * 5;
    if (kind == kInterior) {
      const int wd_ex = ex_local ? S.wd[t.z] : A.wd[t.z];
      if (wd_in == 0 && wd_ex == 0) continue;
      const int gp_in = I, gp_ex = 2 - I;
      double zi, xi, yi, hi, zx, xx, yx, hx;
      side_trace(S, A, in_local, t.y, led_in, gp_in, zi, xi, yi, hi);
      side_trace(S, A, ex_local, t.z, led_ex, gp_ex, zx, xx, yx, hx);
      const int gex = ex_local ? tile0 + t.z : t.z;
      const double sfi = m.sfac_edge ? m.sfac_edge[(size_t)(led_in * 3 + gp_in) * ne + gin] : 1.0;
      const double sfx = m.sfac_edge ? m.sfac_edge[(size_t)(led_ex * 3 + gp_ex) * ne + gex] : 1.0;
      Flux3 f = llf<kNonlin>(P, zi, zx, xi, xx, yi, yx, hi, hx, sfi, sfx, nx, ny, P.g);
      double F = f.f, gi = f.g, hi2 = f.h, gx = f.g, hx2 = f.h;
      // internal_edge_hydro.F:212-302: mass flux out of / into a dry element
      if (fabs(f.f) > 1.0e-8 && (wd_in == 0 || wd_ex == 0)) {
        const double tx = -ny, ty = nx;
        if (wd_in == 0) {
          if (f.f > 0.0) {
            const double qne = xx * nx + yx * ny, qte = xx * tx + yx * ty;
            const double qni = -qne, qti = qte, den = nx * ty - ny * tx;
            const double qxi = (ty * qni - ny * qti) / den, qyi = (-tx * qni + nx * qti) / den;
            Flux3 r = llf<kNonlin>(P, zx, zx, qxi, xx, qyi, yx, hx, hx, sfx, sfx, nx, ny, P.g);
            F = r.f; gx = r.g; hx2 = r.h; gi = 0.0; hi2 = 0.0;
          } else {
            Flux3 r = llf<kNonlin>(P, zi, zx, xi, xx, yi, yx, hi, hx, sfi, sfx, nx, ny, 0.0);
            gi = r.g; hi2 = r.h;
          }
        } else {
          if (f.f < 0.0) {
            const double qni = xi * nx + yi * ny, qti = xi * tx + yi * ty;
            const double qne = -qni, qte = qti, den = nx * ty - ny * tx;
            const double qxe = (ty * qne - ny * qte) / den, qye = (-tx * qne + nx * qte) / den;
            Flux3 r = llf<kNonlin>(P, zi, zi, xi, qxe, yi, qye, hi, hi, sfi, sfi, nx, ny, P.g);
            F = r.f; gi = r.g; hi2 = r.h; gx = 0.0; hx2 = 0.0;
          } else {
            Flux3 r = llf<kNonlin>(P, zi, zx, xi, xx, yi, yx, hi, hx, sfi, sfx, nx, ny, 0.0);
            gx = r.g; hx2 = r.h;
          }
        }
      }
      out[0] = F; out[1] = gi; out[2] = hi2; out[3] = gx; out[4] = hx2;
    } else {
      if (wd_in == 0) continue;
      double zi, xi, yi, hi, zx, xx, yx;
      side_trace(S, A, true, t.y, led_in, I, zi, xi, yi, hi);
      const double sfi = m.sfac_edge ? m.sfac_edge[(size_t)(led_in * 3 + I) * ne + gin] : 1.0;
      ghost_state(A, S.B, kind, t.z, I, zi, xi, yi, hi, nx, ny, zx, xx, yx);
      Flux3 f = llf<kNonlin>(P, zi, zx, xi, xx, yi, yx, hi, hi, sfi, sfi, nx, ny, P.g);
      out[0] = f.f; out[1] = f.g; out[2] = f.h;
    }
  }
  __syncthreads();
  if (!valid) return;

  // ---- phase 3: accumulate in the reference's order, volume, SSP ----
  const BasisP1& B = S.B;
  const int wde = S.wd[tid];
  const double areas = S.geo[0][tid];
  double rhs[9], isum[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) { rhs[c] = 0.0; isum[c] = 0.0; }
#pragma unroll 1
  for (int s = 0; s < 3; ++s) {
    const int l = ei_order(info, s);
    const unsigned kind = ei_kind(info, l);
    if (kind == kNone) continue;
    if (kind == kIBarrier) {
      double o[9];
      ibarrier_side<kNonlin>(A, link[l], (int)ei_flag(info, l) ? 0 : 1, o);
#pragma unroll
      for (int c = 0; c < 9; ++c) rhs[c] = rhs[c] + o[c];
      continue;
    }
    const double xlen = S.geo[1 + 3 * l][tid];
    const double* r = res + (size_t)S.task_of[l][tid] * 15;
    if (kind == kInterior) {
      const int nb = link[l];
      const bool nbr_local = nb >= tile0 && nb < tile0 + ntile;
      const int wdn = nbr_local ? S.wd[nb - tile0] : A.wd[nb];
      if (wde == 0 && wdn == 0) continue;
      const bool is_in = ei_flag(info, l) != 0;
      const double edfac = xlen / areas;
      double acc[9];
#pragma unroll
      for (int c = 0; c < 9; ++c) acc[c] = 0.0;
#pragma unroll 1
      for (int I = 0; I < 3; ++I) {
        const int j = is_in ? I : 2 - I;
        const double* p = r + 5 * I;
        const double F = p[0], Gm = is_in ? p[1] : p[3], Hm = is_in ? p[2] : p[4];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double w = edfac * B.edgeq[l][j][k];
          if (is_in) {  // rhs_*_in(k) = rhs_*_in(k) - w_in * flux
            acc[k] = acc[k] - w * F;
            acc[3 + k] = acc[3 + k] - w * Gm;
            acc[6 + k] = acc[6 + k] - w * Hm;
          } else {      // rhs_*_ex(k) = rhs_*_ex(k) + w_ex * flux
            acc[k] = acc[k] + w * F;
            acc[3 + k] = acc[3 + k] + w * Gm;
            acc[6 + k] = acc[6 + k] + w * Hm;
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 9; ++c) isum[c] = isum[c] + acc[c];
    } else {
      if (wde == 0) continue;
#pragma unroll 1
      for (int I = 0; I < 3; ++I) {
        const double* p = r + 5 * I;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double w = 2.0 * B.m_inv[k] / areas * xlen * B.phi_edge[l][I][k] * B.wegp[I];
          rhs[k] = rhs[k] - w * p[0];
          rhs[3 + k] = rhs[3 + k] - w * p[1];
          rhs[6 + k] = rhs[6 + k] - w * p[2];
        }
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) rhs[c] = rhs[c] + isum[c];  // add_internal_flux

  double q[9], hbe[3];
#pragma unroll
  for (int c = 0; c < 9; ++c) q[c] = S.q[c][tid];
#pragma unroll
  for (int k = 0; k < 3; ++k) hbe[k] = S.q[9 + k][tid];

  // rhs_dg_hydro.F:58-470
  const double area = areas * 0.5;
  const double drdx = 1.0 / area * S.geo[10][tid];
  const double dsdx = 1.0 / area * S.geo[11][tid];
  const double drdy = 1.0 / area * S.geo[12][tid];
  const double dsdy = 1.0 / area * S.geo[13][tid];
  int nd[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) nd[v] = m.nm[(size_t)v * ne + e];
  double xfac[3][3], yfac[3][3];  // [mode][point]
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double dpx = B.drphi[k][i] * drdx + B.dsphi[k][i] * dsdx;
      const double dpy = B.drphi[k][i] * drdy + B.dsphi[k][i] * dsdy;
      xfac[k][i] = B.m_inv[k] * B.wagp[i] * dpx;
      yfac[k][i] = B.m_inv[k] * B.wagp[i] * dpy;
    }
  if (P.rainfall == 1) {
    const double src = 7.0556e-6;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int k = 0; k < 3; ++k) rhs[k] = rhs[k] + B.m_inv[k] * B.wagp[i] * B.phi_area[k][i] * src;
  }
  if (wde != 0) {
    const double NLEQ = kNonlin ? 1.0 : P.nleq, LEQ = kNonlin ? 0.0 : P.leq;
    const double depth_c = hbe[0] + q[0];
    const double fh_c = 1.0 / (kNonlin ? depth_c : NLEQ * depth_c + LEQ);
    const double cori = m.cori ? m.cori[e] : P.cori;
    double fric = m.fric ? m.fric[e] : P.fric;
    double nbar = 0.0;
    if (m.manning) nbar = (m.manning[nd[0]] + m.manning[nd[1]] + m.manning[nd[2]]) / 3.;
    double dpsidx[3] = {0, 0, 0}, dpsidy[3] = {0, 0, 0};
    if (P.nws != 0) {
      const double drpsi[3] = {-0.5, 0.5, 0.0}, dspsi[3] = {-0.5, 0.0, 0.5};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        dpsidx[a] = drpsi[a] * drdx + dspsi[a] * dsdx;
        dpsidy[a] = drpsi[a] * drdy + dspsi[a] * dsdy;
      }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      double zq = q[0], uq = q[3], vq = q[6];
      const double hq = hbe[0] * B.phi_area[0][i] + hbe[1] * B.phi_area[1][i] + hbe[2] * B.phi_area[2][i];
      double dhx = 0.0, dhy = 0.0;
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        dhx = dhx + hbe[k] * (B.drphi[k][i] * drdx + B.dsphi[k][i] * dsdx);
        dhy = dhy + hbe[k] * (B.drphi[k][i] * drdy + B.dsphi[k][i] * dsdy);
      }
      zq = zq + q[1] * B.phi_area[1][i] + q[2] * B.phi_area[2][i];
      uq = uq + q[4] * B.phi_area[1][i] + q[5] * B.phi_area[2][i];
      vq = vq + q[7] * B.phi_area[1][i] + q[8] * B.phi_area[2][i];
      const double depth = zq + hq;
      const double sfq = m.sfac_area ? m.sfac_area[(size_t)i * ne + e] : 1.0;
      const double f1 = kNonlin ? 1.0 : NLEQ + LEQ * hq;
      const double fx = uq * f1 * sfq, fy = vq * f1;
      const double fu = kNonlin ? uq : NLEQ * uq, fv = kNonlin ? vq : NLEQ * vq;
      const double fg = P.nleqg * zq * wde;
      const double fh = 1.0 / (kNonlin ? depth : NLEQ * depth + LEQ);
      const double u = uq * fh, v = vq * fh;
      const double huu = fu * u, hvv = fv * v, huv = fu * v;
      const double gh2 = kNonlin ? fg * (0.5 * zq + hq) : fg * (0.5 * zq + hq) + P.fg_l * zq;
      const double gx = (huu + gh2) * sfq, gy = huv;
      const double hx = huv * sfq, hy = hvv + gh2;
      if (m.manning) {
        fric = P.g * (nbar * nbar) / pow(depth, 1.0 / 3.0);
        if (fric < P.cf) fric = P.cf;
      }
      double tau = fric;
      if (P.iflinbf == 0) {
        const double umag = sqrt(u * u + v * v);
        tau = tau * umag * fh;
        if (P.ifhybf == 1) tau = tau * pow(1.0 + pow(P.hbreak * fh_c, P.ftheta), P.fgamma / P.ftheta);
        tau = fmin(tau, .9 * (1.0 / P.dtdp));
      }
      double sx = -(tau * uq) + fg * dhx * sfq + cori * vq;
      double sy = -(tau * vq) + fg * dhy - cori * uq;
      if (P.nws != 0) {
        // met_forcing.F:49-66: the nodal fields are scaled by the ramp each stage
        const double fw = 1.0 / f1, r = A.rampdg;
        const int n0 = nd[0], n1 = nd[1], n2 = nd[2];
        const double wx0 = r * A.wsx[n0], wx1 = r * A.wsx[n1], wx2 = r * A.wsx[n2];
        const double wy0 = r * A.wsy[n0], wy1 = r * A.wsy[n1], wy2 = r * A.wsy[n2];
        const double p0 = r * A.pr[n0], p1 = r * A.pr[n1], p2 = r * A.pr[n2];
        sx = sx + fw * (wx0 * B.psi[0][i] + wx1 * B.psi[1][i] + wx2 * B.psi[2][i]) -
             P.g * sfq * depth * (p0 * dpsidx[0] + p1 * dpsidx[1] + p2 * dpsidx[2]);
        sy = sy + fw * (wy0 * B.psi[0][i] + wy1 * B.psi[1][i] + wy2 * B.psi[2][i]) -
             P.g * depth * (p0 * dpsidy[0] + p1 * dpsidy[1] + p2 * dpsidy[2]);
      }
      const double sr0 = B.m_inv[0] * B.wagp[i] * B.phi_area[0][i];
      rhs[3] = rhs[3] + sr0 * sx;
      rhs[6] = rhs[6] + sr0 * sy;
#pragma unroll
      for (int k = 1; k < 3; ++k) {
        const double sr = B.m_inv[k] * B.wagp[i] * B.phi_area[k][i];
        rhs[k] = rhs[k] + xfac[k][i] * fx + yfac[k][i] * fy;
        rhs[3 + k] = rhs[3 + k] + xfac[k][i] * gx + yfac[k][i] * gy + sr * sx;
        rhs[6 + k] = rhs[6 + k] + xfac[k][i] * hx + yfac[k][i] * hy + sr * sy;
      }
    }
  }
  if (A.rout) {
#pragma unroll
    for (int c = 0; c < 9; ++c) A.rout[(size_t)c * ne + e] = rhs[c];
  }
  // SSP-RK combination (DG_hydro_timestep.F:238-290); zero coefficients skipped
  bool bad = false;
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    double acc = 0.0;
    for (int I = 0; I < A.irk; ++I) {
      const bool cur = I == A.irk - 1;
      if (A.a[I] != 0.0) acc = acc + A.a[I] * (cur ? q[c] : A.qhist[I][(size_t)c * ne + e]);
      if (A.b[I] != 0.0) acc = acc + A.b[I] * (cur ? rhs[c] : A.rhist[I][(size_t)c * ne + e]);
    }
    bad = bad || isnan(acc);
    A.qout[(size_t)c * ne + e] = acc;
  }
  if (bad) atomicOr(A.err, 1u);
}

// slopelimiter.F:3300-3404: min/max of element means over each node's star
__global__ void node_minmax(const __grid_constant__ LimitArgs L) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= L.m.np) return;
  const int ne = L.m.ne;
  double zmin = 99999., zmax = -99999., xmin = 99999., xmax = -99999., ymin = 99999., ymax = -99999.;
  for (int p = L.m.star_ptr[n]; p < L.m.star_ptr[n + 1]; ++p) {
    const int e = L.m.star[p];
    const double zt = L.q[e], xt = L.q[(size_t)3 * ne + e], yt = L.q[(size_t)6 * ne + e];
    zmin = fmin(zmin, zt); xmin = fmin(xmin, xt); ymin = fmin(ymin, yt);
    zmax = fmax(zmax, zt); xmax = fmax(xmax, xt); ymax = fmax(ymax, yt);
  }
  const int np = L.m.np;
  L.minmax[n] = zmin;
  L.minmax[(size_t)np + n] = zmax;
  L.minmax[(size_t)2 * np + n] = xmin;
  L.minmax[(size_t)3 * np + n] = xmax;
  L.minmax[(size_t)4 * np + n] = ymin;
  L.minmax[(size_t)5 * np + n] = ymax;
}

// slopelimiter.F:3434-3779 (vertex clamp + 3 redistribution sweeps) followed
// by wetdry.F:61-548 for the same element.
__global__ void __launch_bounds__(256) limit_wetdry(const __grid_constant__ LimitArgs L) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = L.m.ne, np = L.m.np;
  if (e >= ne) return;
  const BasisP1& B = cBasis;
  int nd[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) nd[v] = L.m.nm[(size_t)v * ne + e];
  double q[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) q[c] = L.q[(size_t)c * ne + e];
  if (L.slopeflag != 0) {
#pragma unroll
    for (int var = 0; var < 3; ++var) {
      double* zc = &q[3 * var];
      double vmin[3], vmax[3], vx[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        vmin[a] = L.minmax[(size_t)(2 * var) * np + nd[a]];
        vmax[a] = L.minmax[(size_t)(2 * var + 1) * np + nd[a]];
        vx[a] = zc[0] + B.phi_corner[a][1] * zc[1] + B.phi_corner[a][2] * zc[2];
        vx[a] = fmax(fmin(vx[a], vmax[a]), vmin[a]);
      }
#pragma unroll
      for (int sweep = 0; sweep < 3; ++sweep) {
        const double sumloc = (vx[0] + vx[1] + vx[2]) / 3.0;
        double sumdif = (sumloc - zc[0]) * 3.0;
        const double signdif = copysign(1.0, sumdif);
        double dif[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) dif[a] = (vx[a] - zc[0]) * signdif;
        int kdp = (dif[0] > 0) + (dif[1] > 0) + (dif[2] > 0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const double div = fmax(1.0, (double)kdp);
          double redfac = 0.0;
          if (dif[k] > 0) {
            redfac = sumdif * signdif / div;
            kdp = kdp - 1;
          }
          const double redmax = signdif > 0 ? vx[k] - vmin[k] : vmax[k] - vx[k];
          redfac = fmin(redfac, redmax);
          sumdif = sumdif - redfac * signdif;
          vx[k] = vx[k] - redfac * signdif;
        }
      }
      zc[1] = -(1.0 / 6.0 * (vx[0] + vx[1])) + 1.0 / 3.0 * vx[2];
      zc[2] = -(.5 * vx[0]) + .5 * vx[1];
    }
  }
  if (L.wetdry) {
    const double H0 = L.ph.h0, ZERO = 1.0e-6, c13 = 1.0 / 3.0, c16 = 1.0 / 6.0;
    double dpn[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) dpn[v] = L.m.dp[nd[v]];
    const double dpe_min = fmin(fmin(dpn[0], dpn[1]), dpn[2]);
    int wd = L.wd[e];
    int ndry = 0, hmax_i = 0;
    double hmax = ZERO, ht[3], zn[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      zn[v] = q[0] + B.phi_corner[v][1] * q[1] + B.phi_corner[v][2] * q[2];
      ht[v] = dpn[v] + zn[v];
      if (ht[v] > hmax) { hmax_i = v; hmax = ht[v]; }
      if (ht[v] <= H0 + ZERO) ++ndry;
    }
    const double dp_avg = c13 * (dpn[0] + dpn[1] + dpn[2]);
    double zh[3] = {0.0, 0.0, 0.0};
    bool check = false;
    if (ndry == 0) {
      if (wd != 1) {
        zh[0] = zn[0]; zh[1] = zn[1]; zh[2] = zn[2];
        check = true;
      }
    } else {
      const double ht_avg = q[0] + dp_avg;
      if (ndry == 3 || ht_avg <= H0 + ZERO) {  // cases 2 and 3A: flatten, stop flow
        q[0] = ht_avg - dp_avg;
        if (ht_avg < ZERO) q[0] = ZERO - dp_avg;
        q[1] = -L.m.hb[(size_t)ne + e];
        q[2] = -L.m.hb[(size_t)2 * ne + e];
#pragma unroll
        for (int c = 3; c < 9; ++c) q[c] = 0.0;
        if (ndry == 3) {
          wd = 0;
        } else {
          zh[0] = q[0]; zh[1] = q[0]; zh[2] = q[0];
          check = true;
        }
      } else {  // case 3B: move water to the dry vertices, momentum to the wet ones
        int l2h[3] = {0, 1, 2};
#pragma unroll
        for (int k1 = 0; k1 < 3; ++k1)
#pragma unroll
          for (int k2 = k1; k2 < 3; ++k2)
            if (ht[l2h[k1]] > ht[l2h[k2]]) { const int t = l2h[k1]; l2h[k1] = l2h[k2]; l2h[k2] = t; }
        double dh[3];
        dh[l2h[0]] = fmax(H0, ht[l2h[0]]) - ht[l2h[0]];
        dh[l2h[1]] = fmax(H0, ht[l2h[1]] - 0.5 * dh[l2h[0]]) - ht[l2h[1]];
        dh[l2h[2]] = -dh[l2h[0]] - dh[l2h[1]];
        int nd2 = 0;
        double qxs = 0.0, qys = 0.0, hmax2 = 0.0, hh[3], qxn[3], qyn[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) {
          hh[v] = ht[v] + dh[v];
          if (hh[v] > hmax2) { hmax_i = v; hmax2 = hh[v]; }
          qxn[v] = q[3] + B.phi_corner[v][1] * q[4] + B.phi_corner[v][2] * q[5];
          qyn[v] = q[6] + B.phi_corner[v][1] * q[7] + B.phi_corner[v][2] * q[8];
          if (hh[v] <= H0 + 1.0e-10) { ++nd2; qxs = qxs + qxn[v]; qys = qys + qyn[v]; }
        }
        if (nd2 == 3) {
#pragma unroll
          for (int c = 3; c < 9; ++c) q[c] = 0.0;
        } else {
          qxs = qxs / (3.0 - (double)nd2);
          qys = qys / (3.0 - (double)nd2);
          double qxh[3], qyh[3];
#pragma unroll
          for (int v = 0; v < 3; ++v) {
            const bool dry = hh[v] <= H0 + 1.0e-10;
            qxh[v] = dry ? 0.0 : qxn[v] + qxs;
            qyh[v] = dry ? 0.0 : qyn[v] + qys;
          }
          q[3] = c13 * (qxh[0] + qxh[1] + qxh[2]);
          q[4] = -(c16 * (qxh[0] + qxh[1])) + c13 * qxh[2];
          q[5] = -(0.5 * qxh[0]) + 0.5 * qxh[1];
          q[6] = c13 * (qyh[0] + qyh[1] + qyh[2]);
          q[7] = -(c16 * (qyh[0] + qyh[1])) + c13 * qyh[2];
          q[8] = -(0.5 * qyh[0]) + 0.5 * qyh[1];
        }
#pragma unroll
        for (int v = 0; v < 3; ++v) zh[v] = hh[v] - dpn[v];
        q[1] = -(c16 * (zh[0] + zh[1])) + c13 * zh[2];
        q[2] = -(0.5 * zh[0]) + 0.5 * zh[1];
        check = true;
      }
    }
    if (check) {
      if (zh[hmax_i] > (-dpe_min + H0)) {
        wd = 1;
      } else {
#pragma unroll
        for (int c = 3; c < 9; ++c) q[c] = 0.0;
        wd = 0;
      }
    }
    L.wd[e] = wd;
  }
#pragma unroll
  for (int c = 0; c < 9; ++c) L.q[(size_t)c * ne + e] = q[c];
}

// write_results.F:14-170 (modal2nodal) + NODECODE from the wet flags
__global__ void modal2nodal_kernel(MeshView m, const double* __restrict__ q, const int* __restrict__ wd,
                                   double nleq, double leq, double* eta2, double* uu2, double* vv2,
                                   int* nodecode) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.np) return;
  const int ne = m.ne;
  const BasisP1& B = cBasis;
  double area_sum = 0.0;
  int wet = 0;
  for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
    const int e = m.star[p];
    if (wd[e] == 0) continue;
    wet = 1;
    const int a = m.nm[e], b = m.nm[(size_t)ne + e], c = m.nm[(size_t)2 * ne + e];
    const double areas = (m.x[a] - m.x[c]) * (m.y[b] - m.y[c]) + (m.x[c] - m.x[b]) * (m.y[a] - m.y[c]);
    area_sum = area_sum + 0.5 * areas;
  }
  double et = 0.0, uu = 0.0, vv = 0.0;
  for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
    const int e = m.star[p];
    if (wd[e] == 0) continue;
    const int a = m.nm[e], b = m.nm[(size_t)ne + e], c = m.nm[(size_t)2 * ne + e];
    const int K = (a == n) ? 0 : (b == n) ? 1 : 2;
    const double p1 = B.phi_corner[K][1], p2 = B.phi_corner[K][2];
    const double zd = q[e] + p1 * q[(size_t)ne + e] + p2 * q[(size_t)2 * ne + e];
    const double xd = q[(size_t)3 * ne + e] + p1 * q[(size_t)4 * ne + e] + p2 * q[(size_t)5 * ne + e];
    const double yd = q[(size_t)6 * ne + e] + p1 * q[(size_t)7 * ne + e] + p2 * q[(size_t)8 * ne + e];
    const double hd = m.hb[e] + p1 * m.hb[(size_t)ne + e] + p2 * m.hb[(size_t)2 * ne + e];
    const double areas = (m.x[a] - m.x[c]) * (m.y[b] - m.y[c]) + (m.x[c] - m.x[b]) * (m.y[a] - m.y[c]);
    const double w = 0.50 * areas / area_sum;
    const double fh = 1.0 / (nleq * (zd + hd) + leq);
    et = et + w * zd;
    uu = uu + w * xd * fh;
    vv = vv + w * yd * fh;
  }
  if (eta2) eta2[n] = et;
  if (uu2) uu2[n] = uu;
  if (vv2) vv2[n] = vv;
  if (nodecode) nodecode[n] = wet;
}

// Fortran layout ZE(DOFH,NE) <-> state SoA q[c*NE+e] for one variable
__global__ void fortran_to_soa(const double* __restrict__ f, double* __restrict__ q, int ne, int var) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) q[(size_t)(3 * var + k) * ne + e] = f[(size_t)3 * e + k];
}

__global__ void soa_to_fortran(const double* __restrict__ q, double* __restrict__ f, int ne, int var) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) f[(size_t)3 * e + k] = q[(size_t)(3 * var + k) * ne + e];
}

}  // namespace DGSWEM_VARIANT
}  // namespace dgswem
