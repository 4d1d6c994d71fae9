// hydro_kernels.cuh -- sm_100a kernels of one RK stage of the p=1 DG hydro
// step.  Per stage: stage_p1 (tile kernel: edge fluxes once per edge in
// shared memory, volume integral, SSP combination; no atomics) ->
// node_minmax (slope limiter node pass) -> limit_wetdry (limiter element
// pass + WETDRY).  Every arithmetic sequence follows the reference routine
// named in its comment.  Compiled twice (kernels_fast.cu with FMA
// contraction, kernels_strict.cu without), see hydro_device.cuh.
#pragma once

#include <cuda_runtime.h>

#include "cr_math.cuh"
#include "hydro_device.cuh"

#ifndef DGSWEM_VARIANT
#error "define DGSWEM_VARIANT (fast or strict) before including hydro_kernels.cuh"
#endif

namespace dgswem {
namespace DGSWEM_VARIANT {

__constant__ BasisP1 cBasis;

// Arithmetic type of the stage kernel's edge and volume terms: FP64, or
// FP32 in the mixed-precision variant (kernels_mixed.cu), whose state,
// SSP combination, ocean depth-positivity fix, limiter and wet/dry stay FP64.
#ifdef DGSWEM_MIXED
typedef float real;
#else
typedef double real;
#endif
__constant__ BasisT<real> cBasisR;  // cBasis in that type

// RAMPDG of the stage: from device memory in a replayed CUDA graph (whose
// kernel arguments are fixed at capture), else the launch argument
__device__ __forceinline__ double stage_ramp(const StageArgs& A) { return A.ramp ? *A.ramp : A.rampdg; }

// Element geometry rows in the arithmetic type
__device__ __forceinline__ const real* egeo_r(const MeshView& m) {
#ifdef DGSWEM_MIXED
  return m.egeof;
#else
  return m.egeo;
#endif
}

// Physics constants of the stage kernel's terms in the arithmetic type
struct PhysR {
  real g, nleq, leq, nleqg, fg_l, tau_cap, cori, fric, cf;
};
__device__ __forceinline__ PhysR phys_r(const StageArgs& A) {
#ifdef DGSWEM_MIXED
  const PhysF& p = A.pf;
#else
  const Physics& p = A.ph;
#endif
  return PhysR{p.g, p.nleq, p.leq, p.nleqg, p.fg_l, p.tau_cap, p.cori, p.fric, p.cf};
}

// Asynchronous global -> shared copies (cp.async, completion by
// cp.async.wait_all): the data goes straight to shared memory.
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// all but the most recently committed group of this thread's copies complete
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async8_s(unsigned dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4_s(unsigned dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}

// DEPTH**(1.D0/3.D0) of the Manning friction (rhs_dg_hydro.F).  The strict
// variant takes the correctly rounded value of the reference's expression
// (pow_third, cr_math.cuh: IEEE operations only, so the oracle's correctly
// rounded evaluation gives the same bits); the fast variant takes the cube
// root, which differs from it by less than an ulp's worth of the exponent's
// rounding (1/3 is not a double) and costs a fraction of it.
__device__ __forceinline__ double cube_root(double x) {
#ifdef DGSWEM_FAST_MATH
  return cbrt(x);
#else
  return pow_third(x);
#endif
}
__device__ __forceinline__ float cube_root(float x) { return cbrtf(x); }

template <class T>
struct Flux3T {
  T f, g, h;
};
using Flux3 = Flux3T<double>;

// Total depth HT = ZE*NLEQ + HB of numerical_flux.F's flux evaluation.
template <bool kNonlin, class T>
__device__ __forceinline__ T depth(const Physics& P, T ze, T hb) {
  return kNonlin ? ze + hb : ze * T(P.nleq) + hb;
}

// numerical_flux.F:750-914, Local Lax-Friedrichs, in arithmetic type T.
// kNonlin specialises NLEQ=1, LEQ=0 (the products with 1 and sums with 0 it
// removes are exact).  ht_in / ht_ex: the total depths, depth(ze, hb) --
// passed in so that the mixed-precision kernels can supply them from FP32
// depth traces rather than from an FP32 sum of elevation and bathymetry.
template <bool kNonlin, class T>
__device__ __forceinline__ Flux3T<T> llf(const Physics& P, T ze_in, T ze_ex, T qx_in, T qx_ex, T qy_in,
                                         T qy_ex, T hb_in, T hb_ex, T ht_in, T ht_ex, T sf_in, T sf_ex, T nx,
                                         T ny, T G) {
  const T NLEQ = kNonlin ? T(1) : T(P.nleq);
  const T LEQ = kNonlin ? T(0) : T(P.leq);
  const T nleqg = G * NLEQ;
  const T j1 = ze_ex - ze_in, j2 = qx_ex - qx_in, j3 = qy_ex - qy_in;
  T f1, fx1i, fy1i, fh, ui, vi, fx2i, fy2i, fx3i, fy3i;
  {
    f1 = kNonlin ? T(1) : NLEQ + LEQ * hb_in;
    fx1i = qx_in * f1 * sf_in;
    fy1i = qy_in * f1;
    const T fu = kNonlin ? qx_in : NLEQ * qx_in;
    const T fv = kNonlin ? qy_in : NLEQ * qy_in;
    const T fg = nleqg * ze_in;
    fh = T(1) / (kNonlin ? ht_in : NLEQ * ht_in + LEQ);
    ui = qx_in * fh;
    vi = qy_in * fh;
    const T huu = fu * ui, hvv = fv * vi, huv = fu * vi;
    const T gh2 = kNonlin ? fg * (T(0.5) * ze_in + hb_in) : fg * (T(0.5) * ze_in + hb_in) + T(P.fg_l) * ze_in;
    fx2i = (huu + gh2) * sf_in;
    fy2i = huv;
    fx3i = huv * sf_in;
    fy3i = hvv + gh2;
  }
  T fx1e, fy1e, ue, ve, fx2e, fy2e, fx3e, fy3e;
  {
    const T f1e = kNonlin ? T(1) : NLEQ + LEQ * hb_ex;
    fx1e = qx_ex * f1e * sf_ex;
    fy1e = qy_ex * f1e;
    const T fu = kNonlin ? qx_ex : NLEQ * qx_ex;
    const T fv = kNonlin ? qy_ex : NLEQ * qy_ex;
    const T fg = nleqg * ze_ex;
    const T fhe = T(1) / (kNonlin ? ht_ex : NLEQ * ht_ex + LEQ);
    ue = qx_ex * fhe;
    ve = qy_ex * fhe;
    const T huu = fu * ue, hvv = fv * ve, huv = fu * ve;
    const T gh2 = kNonlin ? fg * (T(0.5) * ze_ex + hb_ex) : fg * (T(0.5) * ze_ex + hb_ex) + T(P.fg_l) * ze_ex;
    fx2e = (huu + gh2) * sf_ex;
    fy2e = huv;
    fx3e = huv * sf_ex;
    fy3e = hvv + gh2;
  }
  const T f1a = T(0.5) * ((fx1i + fx1e) * nx + (fy1i + fy1e) * ny);
  const T f2a = T(0.5) * ((fx2i + fx2e) * nx + (fy2i + fy2e) * ny);
  const T f3a = T(0.5) * ((fx3i + fx3e) * nx + (fy3i + fy3e) * ny);
  const T uni = kNonlin ? ui * nx + vi * ny : (ui * nx + vi * ny) * NLEQ;
  const T nxsi = nx * sf_in, nxse = nx * sf_ex;
  const T ci = sqrt(G * ht_in * (ny * ny + nxsi * nxsi));
  const T une = kNonlin ? ue * nx + ve * ny : (ue * nx + ve * ny) * NLEQ;
  const T ce = sqrt(G * ht_ex * (ny * ny + nxse * nxse));
  // max(|un+c|, |un|, |un-c|) over both sides.  For c >= 0 the rounded
  // |un| + c equals the rounded larger of |un + c| and |un - c| exactly, so
  // fmax(|un| + c, |un|) is the same value; with c = NaN (negative depth) both
  // forms reduce to |un|, as fmax skips NaN operands.
  const T ai = fabs(uni), ae = fabs(une);
  const T eig = fmax(fmax(ai + ci, ai), fmax(ae + ce, ae));
  Flux3T<T> r;
  r.f = f1a - T(0.5) * eig * j1;
  if (kNonlin) {
    r.g = f2a - T(0.5) * eig * j2;
    r.h = f3a - T(0.5) * eig * j3;
  } else {
    const T nx2 = NLEQ + LEQ * nx * nx, ny2 = NLEQ + LEQ * ny * ny, nxy = nx * ny;
    r.g = f2a - T(0.5) * eig * (j2 * nx2 + LEQ * j3 * nxy);
    r.h = f3a - T(0.5) * eig * (j3 * ny2 + LEQ * j2 * nxy);
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
// The ocean elevation sum and its depth-positivity fix are FP64 in every
// variant.
__device__ __forceinline__ void ghost_state(const StageArgs& A, unsigned kind, int list, int j, real zi, real xi,
                                            real yi, real hbi, real nx, real ny, real& zx, real& xx, real& yx) {
  const Physics& P = A.ph;
  const real tx = -ny, ty = nx;
  zx = zi;
  xx = xi;
  yx = yi;
  if (kind == kOcean) {
    // endpoint values EMO*RFF*COS(ARGJ-EFA) come from the host for this stage
    double zsum = 0.0;
    for (int f = 0; f < A.m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * A.m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * cBasis.xegp[j]);
    }
    const double hbd = hbi;
    if (zsum * P.ifnlfa + hbd <= 0) zsum = fabs(hbd) + P.h0;
    zx = (real)zsum;
  } else if (kind == kLand) {
    const real qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const real qne = -qn, qte = qt, den = real(1) / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  } else if (kind == kFlow) {
    // per-point terms QNAM_GP*RFF*COS(ARG) come from the host for this stage
    real qne = 0;
    xx = 0;
    yx = 0;
    for (int f = 0; f < A.m.nffr; ++f) {
      qne = qne + (real)A.flow_qn[((size_t)f * A.m.nfeds + list) * 3 + j];
      xx = -(ty * qne - ny * real(0)) / (nx * ty - ny * tx);
      yx = -(-tx * qne + nx * real(0)) / (nx * ty - ny * tx);
    }
  } else if (kind == kRadiation) {
    const real qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const real qne = -qn + real(2) * sqrt(real(P.g) / (hbi + zi)) * zi, qte = qt,
               den = real(1) / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  } else if (kind == kEBarrier) {
    const real above = zi - (real)A.m.ebht[list];
    const real subsup = real(2) * above / real(3);
    real qne, qte;
    if (above < real(0.01)) {
      qne = -(xi * nx + yi * ny);
      qte = xi * tx + yi * ty;
    } else {
      qne = (real)stage_ramp(A) * (real)A.m.ebcfsp[list] * subsup * sqrt(subsup * real(P.g));
      qte = 0;
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
    const double htb = depth<kNonlin>(P, zeb, hbbp), htf = depth<kNonlin>(P, zef, hbfp);
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
        qfn = (aboveb > ssf) ? stage_ramp(A) * m.ibcfsb[seg] * aboveb * sqrt(2.0 * P.g * (abovef - aboveb))
                             : stage_ramp(A) * m.ibcfsp[seg] * ssf * sqrt(ssf * P.g);
      } else if (aboveb > abovef && aboveb > 0.01) {
        weir = -1;
        qbn = (abovef > ssb) ? stage_ramp(A) * m.ibcfsb[seg] * abovef * sqrt(2.0 * P.g * (aboveb - abovef))
                             : stage_ramp(A) * m.ibcfsp[seg] * ssb * sqrt(ssb * P.g);
      }
    }
    Flux3 fb{0, 0, 0}, ff{0, 0, 0};
    double qxe = 0.0, qye = 0.0;
    bool done = false;
    if (weir <= 0) {
      qxe = (tyb * qbn - nyb * qbt) / (nxb * tyb - nyb * txb);
      qye = (-txb * qbn + nxb * qbt) / (nxb * tyb - nyb * txb);
      fb = llf<kNonlin>(P, zeb, zeb, qxb, qxe, qyb, qye, hbbp, hbbp, htb, htb, sfb, sfb, nxb, nyb, P.g);
      if (weir < 0) {  // the front side keeps the back side's exterior momentum
        ff = llf<kNonlin>(P, zef, zef, qxf, qxe, qyf, qye, hbfp, hbfp, htf, htf, sff, sff, nxf, nyf,
                          wdf == 0 ? 0.0 : P.g);
        done = true;
      }
    }
    if (!done && weir >= 0) {
      qxe = (tyf * qfn - nyf * qft) / (nxf * tyf - nyf * txf);
      qye = (-txf * qfn + nxf * qft) / (nxf * tyf - nyf * txf);
      ff = llf<kNonlin>(P, zef, zef, qxf, qxe, qyf, qye, hbfp, hbfp, htf, htf, sff, sff, nxf, nyf, P.g);
      if (weir > 0)
        fb = llf<kNonlin>(P, zeb, zeb, qxb, qxe, qyb, qye, hbbp, hbbp, htb, htb, sfb, sfb, nxb, nyb,
                          wdb == 0 ? 0.0 : P.g);
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

// Internal-barrier sides of one stage, one thread per (segment, side), into
// ib_rhs[(2*seg + side)*9 + c]; the stage kernel adds them at the edge's
// place in each element's sum.  Runs before stage_p1 on the same stream
// (both only read the stage's input state).  Segments without an opposite
// edge (ib_elem < 0) are skipped, as in the reference.
template <bool kNonlin>
__global__ void __launch_bounds__(128) ibarrier_sides(const __grid_constant__ StageArgs A) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= 2 * A.m.nibseg) return;
  const int seg = w >> 1, side = w & 1;
  if (A.m.ib_elem[2 * seg] < 0) return;
  ibarrier_side<kNonlin>(A, seg, side, A.ib_rhs + (size_t)w * 9);
}

// ---------------------------------------------------------------------------
// Tile stage kernel.  Block b owns tile b of the tile plan built at create:
// up to kTile consecutive elements (the shape's tile), and for them the edge
// tasks the tile evaluates (boundary edges, edges to out-of-tile elements,
// shared interior edges once) and the halo of out-of-tile neighbours those
// tasks read.  Four phases separated by barriers, each spread over all
// kStageThreads threads:
//   1. tile and halo elements: modal state, bathymetry modes and wet/dry flag
//      into shared memory; tile elements also their geometry;
//   2. one thread per (element, area point): volume fluxes and sources (tile
//      elements only: in the FP64 variants the halo's copies are still in
//      flight, waited for at the end of this phase);
//   3. one thread per (task, Lobatto point): the LLF flux of an edge point in
//      the reference's own in/ex orientation with its dry-side rules ->
//      F, G_in, H_in, G_ex, H_ex (internal-barrier sides come from
//      ibarrier_sides);
//   4. one thread per (element, mode): that mode of the three variables
//      summed in the reference's order (boundary edges, interior edges in
//      edge-number order as the slot sum of add_internal_flux, rain, area
//      points), then the SSP combination.
// internal_edge_hydro.F, *_edge_hydro.F, rhs_dg_hydro.F, DG_hydro_timestep.F:238-290
// ---------------------------------------------------------------------------

// resident stage threads per SM the register allocation targets (FP64: two
// blocks of 384, at most 85 registers a thread); a shape of T threads per
// block is compiled for that many over T resident blocks
#ifndef DGSWEM_STAGE_RESIDENT_THREADS
#define DGSWEM_STAGE_RESIDENT_THREADS 768
#endif
constexpr int stage_min_blocks(int threads) {
  return DGSWEM_STAGE_RESIDENT_THREADS / threads > 0 ? DGSWEM_STAGE_RESIDENT_THREADS / threads : 1;
}

// The 12 modal values (ZE, QX, QY, HB modes, contiguous) of shared-memory
// slot `slot` in the arithmetic type: the FP64 slots qs (stride kQStride),
// or their FP32 copy (stride kQfStride) in the mixed variant.
__device__ __forceinline__ void slot_values(const real* qt, int slot, real v[12]) {
#ifdef DGSWEM_MIXED
  const float4* q = reinterpret_cast<const float4*>(qt + slot * kQfStride);
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    const float4 t = q[j];
    v[4 * j] = t.x; v[4 * j + 1] = t.y; v[4 * j + 2] = t.z; v[4 * j + 3] = t.w;
  }
#else
  const double2* q = reinterpret_cast<const double2*>(qt + slot * kQStride);
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    const double2 t = q[j];
    v[2 * j] = t.x; v[2 * j + 1] = t.y;
  }
#endif
}

// Trace at edge point (led, gp) of slot `slot`'s ZE, QX, QY and HB; mode 0
// of the basis is 1 on every edge point.
__device__ __forceinline__ void slot_trace(const BasisT<real>& B, const real* qt, int slot, int led, int gp,
                                           real& z, real& u, real& v, real& h) {
  const real p1 = B.phi_edge[led][gp][1], p2 = B.phi_edge[led][gp][2];
  real q[12];
  slot_values(qt, slot, q);
  z = q[0] + q[1] * p1 + q[2] * p2;
  u = q[3] + q[4] * p1 + q[5] * p2;
  v = q[6] + q[7] * p1 + q[8] * p2;
  h = q[9] + q[10] * p1 + q[11] * p2;
}

// One Lobatto point of an interior edge in the reference's in/ex orientation
// (internal_edge_hydro.F): the LLF flux of the two traces, then the dry-side
// rules of :212-302 -> o[0..4] = F, G_in, H_in, G_ex, H_ex.
template <bool kNonlin>
__device__ __forceinline__ void interior_point(const Physics& P, real zi, real zx, real xi, real xx, real yi,
                                           real yx, real hi, real hx, real hti, real htx, real sfi, real sfx,
                                           real nx, real ny, int wd_in, int wd_ex, real* o) {
  const Flux3T<real> f =
      llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hx, hti, htx, sfi, sfx, nx, ny, real(P.g));
  o[0] = f.f; o[1] = f.g; o[2] = f.h; o[3] = f.g; o[4] = f.h;
  if ((wd_in == 0 || wd_ex == 0) && fabs(f.f) > real(1.0e-8)) {
    // internal_edge_hydro.F:212-302: mass flux out of / into a dry
    // element.  The four cases re-evaluate the flux once with changed
    // arguments: the dry side's state replaced by the wet side's with
    // reflected momentum (outflow from a dry element), or gravity off
    // (G = 0) for the dry side's momentum flux.
    const bool in_dry = wd_in == 0;
    const real F0 = f.f;
    const real tx = -ny, ty = nx, den = nx * ty - ny * tx;
    const bool reflect = in_dry ? F0 > real(0) : F0 < real(0);
    // the wet side, whose momentum is reflected onto the dry side
    const real qxw = in_dry ? xx : xi, qyw = in_dry ? yx : yi;
    const real qnw = qxw * nx + qyw * ny, qtw = qxw * tx + qyw * ty;
    const real qnr = -qnw, qtr = qtw;
    const real qxr = (ty * qnr - ny * qtr) / den, qyr = (-tx * qnr + nx * qtr) / den;
    real a_zi = zi, a_zx = zx, a_xi = xi, a_xx = xx, a_yi = yi, a_yx = yx;
    real a_hi = hi, a_hx = hx, a_ti = hti, a_tx = htx, a_si = sfi, a_sx = sfx, a_g = 0;
    if (reflect) {
      a_g = real(P.g);
      if (in_dry) {
        a_zi = zx; a_xi = qxr; a_yi = qyr; a_hi = hx; a_ti = htx; a_si = sfx;
      } else {
        a_zx = zi; a_xx = qxr; a_yx = qyr; a_hx = hi; a_tx = hti; a_sx = sfi;
      }
    }
    const Flux3T<real> r = llf<kNonlin, real>(P, a_zi, a_zx, a_xi, a_xx, a_yi, a_yx, a_hi, a_hx, a_ti, a_tx,
                                              a_si, a_sx, nx, ny, a_g);
    if (reflect) {
      o[0] = r.f;
      if (in_dry) { o[3] = r.g; o[4] = r.h; o[1] = 0; o[2] = 0; }
      else        { o[1] = r.g; o[2] = r.h; o[3] = 0; o[4] = 0; }
    } else {
      if (in_dry) { o[1] = r.g; o[2] = r.h; }
      else        { o[3] = r.g; o[4] = r.h; }
    }
  }
}

// Bathymetry hb and total depth ht at a trace point from elevation z and the
// slot's fourth trace w: w is HB in the FP64 kernels; the mixed kernels'
// FP32 slots hold the depth modes ZE + HB (summed in FP64, then rounded), so
// that a thin water column keeps FP32 relative accuracy instead of being the
// difference of two rounded values of metres.
template <bool kNonlin>
__device__ __forceinline__ void trace_depth(const Physics& P, real z, real w, real& hb, real& ht) {
#ifdef DGSWEM_MIXED
  hb = w - z;
  ht = kNonlin ? w : depth<kNonlin>(P, z, hb);
#else
  hb = w;
  ht = depth<kNonlin>(P, z, hb);
#endif
}

// Volume fluxes and sources at area point I of element e (rhs_dg_hydro.F:
// 58-470) from the element's 12 slot values q (ZE, QX, QY modes, then HB or,
// in the mixed variant, depth modes), its inverse Jacobian, element-mean
// Manning n and hybrid friction factor: out = fx fy gx gy hx hy sx sy.
template <bool kNonlin, bool kSph>
__device__ __forceinline__ void volume_core(const StageArgs& A, const BasisT<real>& C, const real q[12], real drdx,
                                            real dsdx, real drdy, real dsdy, real nbar, real hyb, int I, int e,
                                            real out[8]) {
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const PhysR R = phys_r(A);
  const int ne = m.ne;
  const int wde = 1;  // volume terms are evaluated for wet elements only
#ifdef DGSWEM_MIXED
  // the slot holds the depth modes ZE + HB (see trace_depth)
  const real hbe[3] = {q[9] - q[0], q[10] - q[1], q[11] - q[2]};
#else
  const real* hbe = q + 9;
#endif
  const real NLEQ = kNonlin ? real(1) : R.nleq, LEQ = kNonlin ? real(0) : R.leq;
  const real cori = m.cori ? (real)m.cori[e] : R.cori;
  real fric = m.fric ? (real)m.fric[e] : R.fric;
  real zq = q[0], uq = q[3], vq = q[6];
  const real hq = hbe[0] * C.phi_area[0][I] + hbe[1] * C.phi_area[1][I] + hbe[2] * C.phi_area[2][I];
  real dhx = 0, dhy = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    dhx = dhx + hbe[k] * (C.drphi[k][I] * drdx + C.dsphi[k][I] * dsdx);
    dhy = dhy + hbe[k] * (C.drphi[k][I] * drdy + C.dsphi[k][I] * dsdy);
  }
  zq = zq + q[1] * C.phi_area[1][I] + q[2] * C.phi_area[2][I];
  uq = uq + q[4] * C.phi_area[1][I] + q[5] * C.phi_area[2][I];
  vq = vq + q[7] * C.phi_area[1][I] + q[8] * C.phi_area[2][I];
#ifdef DGSWEM_MIXED
  const real depth =
      kNonlin ? q[9] + q[10] * C.phi_area[1][I] + q[11] * C.phi_area[2][I] : zq + hq;
#else
  const real depth = zq + hq;
#endif
  const real sfq = kSph ? (real)m.sfac_area[(size_t)I * ne + e] : real(1);
  const real f1 = kNonlin ? real(1) : NLEQ + LEQ * hq;
  const real fx = uq * f1 * sfq, fy = vq * f1;
  const real fu = kNonlin ? uq : NLEQ * uq, fv = kNonlin ? vq : NLEQ * vq;
  const real fg = R.nleqg * zq * wde;
  const real fh = real(1) / (kNonlin ? depth : NLEQ * depth + LEQ);
  const real u = uq * fh, v = vq * fh;
  const real huu = fu * u, hvv = fv * v, huv = fu * v;
  const real gh2 = kNonlin ? fg * (real(0.5) * zq + hq) : fg * (real(0.5) * zq + hq) + R.fg_l * zq;
  const real gx = (huu + gh2) * sfq, gy = huv;
  const real hx = huv * sfq, hy = hvv + gh2;
  if (m.manning) {
    fric = R.g * (nbar * nbar) / cube_root(depth);
    if (fric < R.cf) fric = R.cf;
  }
  real tau = fric;
  if (P.iflinbf == 0) {
    const real umag = sqrt(u * u + v * v);
    tau = tau * umag * fh;
    if (P.ifhybf == 1) tau = tau * hyb;
    tau = fmin(tau, R.tau_cap);
  }
  real sx = -(tau * uq) + fg * dhx * sfq + cori * vq;
  real sy = -(tau * vq) + fg * dhy - cori * uq;
  if (P.nws != 0) {
    // met_forcing.F:49-66: the nodal fields are scaled by the ramp each stage
    const real drpsi[3] = {-0.5, 0.5, 0.0}, dspsi[3] = {-0.5, 0.0, 0.5};
    real dpsidx[3], dpsidy[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dpsidx[a] = drpsi[a] * drdx + dspsi[a] * dsdx;
      dpsidy[a] = drpsi[a] * drdy + dspsi[a] * dsdy;
    }
    const real fw = real(1) / f1, r = (real)stage_ramp(A);
    const int n0 = m.nm[e], n1 = m.nm[(size_t)ne + e], n2 = m.nm[(size_t)2 * ne + e];
    const real wx0 = r * (real)A.wsx[n0], wx1 = r * (real)A.wsx[n1], wx2 = r * (real)A.wsx[n2];
    const real wy0 = r * (real)A.wsy[n0], wy1 = r * (real)A.wsy[n1], wy2 = r * (real)A.wsy[n2];
    const real p0 = r * (real)A.pr[n0], p1 = r * (real)A.pr[n1], p2 = r * (real)A.pr[n2];
    sx = sx + fw * (wx0 * C.psi[0][I] + wx1 * C.psi[1][I] + wx2 * C.psi[2][I]) -
         R.g * sfq * depth * (p0 * dpsidx[0] + p1 * dpsidx[1] + p2 * dpsidx[2]);
    sy = sy + fw * (wy0 * C.psi[0][I] + wy1 * C.psi[1][I] + wy2 * C.psi[2][I]) -
         R.g * depth * (p0 * dpsidy[0] + p1 * dpsidy[1] + p2 * dpsidy[2]);
  }
  out[0] = fx; out[1] = fy; out[2] = gx; out[3] = gy;
  out[4] = hx; out[5] = hy; out[6] = sx; out[7] = sy;
}

// Phase 3 of the stage kernel for area point I of tile element el (global
// id e): volume_core on the element's shared-memory slot and geometry rows,
// into vol[(v*3 + I)*kTile + el] by volume_point.  C: the basis tables in
// shared memory (I is a runtime index); qt: the slots in the arithmetic type.
template <bool kNonlin, bool kSph, int kTile>
__device__ __forceinline__ void volume_values(const StageArgs& A, const BasisT<real>& C, const real* qt,
                                              const real* geo, int I, int el, int e, real out[8]) {
  real q[12];
  slot_values(qt, el, q);
  const real drdx = geo[EGeo::kDrdx * kTile + el], dsdx = geo[EGeo::kDsdx * kTile + el];
  const real drdy = geo[EGeo::kDrdy * kTile + el], dsdy = geo[EGeo::kDsdy * kTile + el];
  const real nbar = A.m.manning ? geo[EGeo::kNbar * kTile + el] : real(0);
  const real hyb = (A.ph.iflinbf == 0 && A.ph.ifhybf == 1) ? geo[SGeo::kHyb * kTile + el] : real(0);
  volume_core<kNonlin, kSph>(A, C, q, drdx, dsdx, drdy, dsdy, nbar, hyb, I, e, out);
}

template <bool kNonlin, bool kSph, int kTile>
__device__ __forceinline__ void volume_point(const StageArgs& A, const BasisT<real>& C, const real* qt,
                                             const real* geo, real* vol, int I, int el, int e) {
  real v[8];
  volume_values<kNonlin, kSph, kTile>(A, C, qt, geo, I, el, e, v);
#pragma unroll
  for (int r = 0; r < 8; ++r) vol[(r * 3 + I) * kTile + el] = v[r];
}

// Phase 4 of the stage kernel for mode K of tile element el (global id e):
// the right-hand side of mode K of the three variables, each summed in the
// reference's order -- boundary edges, interior edges in edge-number order
// (the slot sum of add_internal_flux), rain, area points -- then the SSP
// combination (DG_hydro_timestep.F:238-290) written to qout.  The edge and
// area-point weights of mode K are formed once for the three variables.  The
// basis tables come from constant memory (cBasisR): K is the same for a
// whole warp and the point indices are fixed by unrolled loops; the edge
// weights' per-lane (edge, point) rows cost a few distinct addresses a warp
// but keep the load off the shared-memory pipe.  The sums are in the arithmetic
// type, the SSP combination in FP64 (in the mixed variant: the RHS rounded
// to FP32, the stage states and their combination FP64).
template <bool kNonlin, int kTile>
__device__ __forceinline__ void sum_mode(const StageArgs& A, const double* qs,
                                         const real* geo, const real* vol, const real* res, const int* tdry,
                                         const unsigned* sinfo, const int* wds, const uint2* stasks, int K, int el,
                                         int e) {
  const BasisT<real>& C = cBasisR;
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const int ne = m.ne;
  // SSP terms of stage 1 fetched first so that their latency overlaps the
  // sums below; the combination keeps the reference's order
  const bool hist0 = A.irk > 1;
  double h0q[3] = {0.0, 0.0, 0.0}, h0r[3] = {0.0, 0.0, 0.0};
  if (hist0) {
#pragma unroll
    for (int V = 0; V < 3; ++V) {
      const size_t c = (size_t)(3 * V + K) * ne + e;
      if (A.a[0] != 0.0) h0q[V] = A.qhist[0][c];
      if (A.b[0] != 0.0) h0r[V] = A.rhist[0][c];
    }
  }
  const unsigned info = sinfo[el], slots = sinfo[kTile + el];
  const int wde = wds[el];
  real rhs[3] = {0, 0, 0}, isum[3] = {0, 0, 0};
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int l = ei_order(info, s);
    const unsigned kind = ei_kind(info, l);
    if (kind == kNone) continue;
    const int ti = (slots >> (10 * l)) & kNoTask;
    const real* r = res + (size_t)ti * 15;
    if (kind == kIBarrier) {
      const double* o = A.ib_rhs + (size_t)stasks[ti].y * 9;
#pragma unroll
      for (int V = 0; V < 3; ++V) rhs[V] = rhs[V] + (real)o[3 * V + K];
      continue;
    }
    if (kind == kInterior) {
      if (tdry[ti]) continue;
      const bool is_in = ei_flag(info, l) != 0;
      const int c1 = is_in ? 1 : 3;  // G and H of this side: components c1, c1 + 1
      const real edfac = geo[(EGeo::kEdfac + l) * kTile + el];
      real acc[3] = {0, 0, 0};
#pragma unroll
      for (int I = 0; I < 3; ++I) {
        const int j = is_in ? I : 2 - I;
        const real wk = edfac * C.edgeq[l][j][K];  // constant memory: off the shared-memory pipe
        const real* rv = r + 5 * I;
        const real val[3] = {rv[0], rv[c1], rv[c1 + 1]};
#pragma unroll
        for (int V = 0; V < 3; ++V) {
          if (is_in)  // rhs_*_in(k) = rhs_*_in(k) - w_in * flux
            acc[V] = acc[V] - wk * val[V];
          else        // rhs_*_ex(k) = rhs_*_ex(k) + w_ex * flux
            acc[V] = acc[V] + wk * val[V];
        }
      }
#pragma unroll
      for (int V = 0; V < 3; ++V) isum[V] = isum[V] + acc[V];
    } else {
      if (wde == 0) continue;
      const real areas = egeo_r(m)[(size_t)EGeo::kAreas * ne + e];
      const real xlen = egeo_r(m)[(size_t)(EGeo::kXlen + l) * ne + e];
#pragma unroll
      for (int I = 0; I < 3; ++I) {
        const real wk = real(2) * C.m_inv[K] / areas * xlen * C.phi_edge[l][I][K] * C.wegp[I];
#pragma unroll
        for (int V = 0; V < 3; ++V) rhs[V] = rhs[V] - wk * r[5 * I + V];
      }
    }
  }
#pragma unroll
  for (int V = 0; V < 3; ++V) rhs[V] = rhs[V] + isum[V];  // add_internal_flux
  if (P.rainfall == 1) {
    const real src = real(7.0556e-6);
#pragma unroll
    for (int i = 0; i < 3; ++i) rhs[0] = rhs[0] + C.srfac[K][i] * src;
  }
  if (wde != 0) {
    const real drdx = geo[EGeo::kDrdx * kTile + el], dsdx = geo[EGeo::kDsdx * kTile + el];
    const real drdy = geo[EGeo::kDrdy * kTile + el], dsdy = geo[EGeo::kDsdy * kTile + el];
    // vol rows: fx fy gx gy hx hy sx sy, each [point][tile]
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const real sr = C.srfac[K][i];
      const real sx = vol[(6 * 3 + i) * kTile + el], sy = vol[(7 * 3 + i) * kTile + el];
      if (K == 0) {
        rhs[1] = rhs[1] + sr * sx;
        rhs[2] = rhs[2] + sr * sy;
      } else {
        const real dpx = C.drphi[K][i] * drdx + C.dsphi[K][i] * dsdx;
        const real dpy = C.drphi[K][i] * drdy + C.dsphi[K][i] * dsdy;
        const real xf = C.mw[K][i] * dpx;
        const real yf = C.mw[K][i] * dpy;
        const real fx = vol[(0 * 3 + i) * kTile + el], fy = vol[(1 * 3 + i) * kTile + el];
        const real gx = vol[(2 * 3 + i) * kTile + el], gy = vol[(3 * 3 + i) * kTile + el];
        const real hx = vol[(4 * 3 + i) * kTile + el], hy = vol[(5 * 3 + i) * kTile + el];
        rhs[0] = rhs[0] + xf * fx + yf * fy;
        rhs[1] = rhs[1] + xf * gx + yf * gy + sr * sx;
        rhs[2] = rhs[2] + xf * hx + yf * hy + sr * sy;
      }
    }
  }
  // SSP-RK combination (DG_hydro_timestep.F:238-290); zero coefficients skipped
  bool bad = false;
#pragma unroll
  for (int V = 0; V < 3; ++V) {
    const int c = 3 * V + K;
    const double rk = (double)rhs[V];
    if (A.rout) A.rout[(size_t)c * ne + e] = rk;
    const double qc = qs[el * kQStride + c];
    double acc = 0.0;
    if (hist0) {
      if (A.a[0] != 0.0) acc = acc + A.a[0] * h0q[V];
      if (A.b[0] != 0.0) acc = acc + A.b[0] * h0r[V];
    }
    for (int I = 1; I < A.irk; ++I) {
      const bool cur = I == A.irk - 1;
      if (A.a[I] != 0.0) acc = acc + A.a[I] * (cur ? qc : A.qhist[I][(size_t)c * ne + e]);
      if (A.b[I] != 0.0) acc = acc + A.b[I] * (cur ? rk : A.rhist[I][(size_t)c * ne + e]);
    }
    if (!hist0) {  // stage 1: the current stage is I = 0
      if (A.a[0] != 0.0) acc = acc + A.a[0] * qc;
      if (A.b[0] != 0.0) acc = acc + A.b[0] * rk;
    }
    bad = bad || isnan(acc);
    A.qout[(size_t)c * ne + e] = acc;
  }
  if (bad) atomicOr(A.err, 1u);
}

template <bool kNonlin, bool kSph, int kTile, int kStageThreads>
__global__ void __launch_bounds__(kStageThreads, stage_min_blocks(kStageThreads))
    stage_p1(const __grid_constant__ StageArgs A) {
  static_assert(kTile % 32 == 0 && kStageThreads % kTile == 0 && kStageThreads > kTile, "tile shape");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const int ne = m.ne;
  const int tid = threadIdx.x;
  const int tile = A.tile_list ? A.tile_list[A.tile_off + (int)blockIdx.x] : (int)blockIdx.x;
  const int tile0 = m.tile_elem_ptr[tile];
  const int n = m.tile_elem_ptr[tile + 1] - tile0;
  const int hbeg = m.tile_halo_ptr[tile], nh = m.tile_halo_ptr[tile + 1] - hbeg;
  const int tbeg = m.tile_task_ptr[tile], ntask = m.tile_task_ptr[tile + 1] - tbeg;
  const StageLayout L = stage_layout(kTile, m.max_halo, m.max_tasks, (unsigned)sizeof(real));
  double* qs = reinterpret_cast<double*>(smem_raw + L.qs);
  real* geo = reinterpret_cast<real*>(smem_raw + L.geo);
#ifdef DGSWEM_MIXED
  real* qt = reinterpret_cast<real*>(smem_raw + L.qf);  // FP32 copy of the slots
#else
  const real* qt = qs;
#endif
  real* vol = reinterpret_cast<real*>(smem_raw + L.vol);
  real* res = reinterpret_cast<real*>(smem_raw + L.res);
  int* wds = reinterpret_cast<int*>(smem_raw + L.wd);
  int* gid = reinterpret_cast<int*>(smem_raw + L.gid);
  int* tdry = reinterpret_cast<int*>(smem_raw + L.tdry);
  unsigned* sinfo = reinterpret_cast<unsigned*>(smem_raw + L.info);  // [einfo | eslot][kTile]
  uint2* stasks = reinterpret_cast<uint2*>(smem_raw + L.tasks);      // the tile's edge-task words

  // ---- phase 1: tile and halo elements into shared memory ----
#ifdef DGSWEM_MIXED
  // Thread w < kTile: tile element w's 12 modal values (state rows and
  // bathymetry rows; consecutive threads on consecutive elements of a row)
  // into registers, then its FP32 slot and the FP64 state the SSP
  // combination reads.  The other threads: the geometry rows and flags
  // (cp.async) and the halo elements' FP32 slots, one thread per element.
  {
    static_assert(kStageThreads > kTile && (kStageThreads - kTile) % kTile == 0,
                  "geometry rows are copied by whole groups of kTile threads");
    if (tid < kTile) {
      if (tid < n) {
        double v[12];
        const double* src = A.qin + tile0 + tid;
#pragma unroll
        for (int r = 0; r < 9; ++r) v[r] = src[(size_t)r * ne];
        src = m.hb + tile0 + tid;
#pragma unroll
        for (int k = 0; k < 3; ++k) v[9 + k] = src[(size_t)k * ne];
        double2* d = reinterpret_cast<double2*>(qs + tid * kQStride);
#pragma unroll
        for (int j = 0; j < 5; ++j) d[j] = make_double2(v[2 * j], v[2 * j + 1]);
        // FP32 slot: ZE, QX, QY modes and the depth modes ZE + HB (FP64 sums)
#pragma unroll
        for (int k = 0; k < 3; ++k) v[9 + k] = v[k] + v[9 + k];
        float4* f = reinterpret_cast<float4*>(qt + tid * kQfStride);
#pragma unroll
        for (int j = 0; j < 3; ++j)
          f[j] = make_float4((float)v[4 * j], (float)v[4 * j + 1], (float)v[4 * j + 2], (float)v[4 * j + 3]);
        // hybrid friction factor from the element-mean depth (depth mode 1)
        if (P.iflinbf == 0 && P.ifhybf == 1) {
          const real depth_c = (real)v[9];
          const real fh_c = real(1) / (kNonlin ? depth_c : real(P.nleq) * depth_c + real(P.leq));
          geo[SGeo::kHyb * kTile + tid] =
              pow(real(1) + pow(real(P.hbreak) * fh_c, real(P.ftheta)), real(P.fgamma / P.ftheta));
        }
      }
    } else {
      constexpr int kU = kStageThreads - kTile, kStep = kU / kTile;
      const int u = tid - kTile, w = u % kTile, r0 = u / kTile;
      if (w < n) {
        const int ngeo = m.manning ? EGeo::kSmemRows : EGeo::kNbar;
        const size_t step = (size_t)kStep * ne;
        const unsigned gdst = smem_addr(geo) + (unsigned)(r0 * kTile + w) * 4u;
        const real* gsrc = egeo_r(m) + (size_t)r0 * ne + tile0 + w;
#pragma unroll
        for (int j = 0; j < (EGeo::kSmemRows + kStep - 1) / kStep; ++j)
          if (r0 + j * kStep < ngeo) cp_async4_s(gdst + 4u * kStep * kTile * j, gsrc + j * step);
#pragma unroll
        for (int j = 0; j < (3 + kStep - 1) / kStep; ++j) {
          const int r = r0 + j * kStep;
          if (r == 0)
            cp_async4(wds + w, A.wd + tile0 + w);
          else if (r < 3)
            cp_async4(sinfo + (r - 1) * kTile + w, (r == 1 ? m.einfo : m.eslot) + tile0 + w);
        }
      }
      for (int j = u; j < ntask; j += kU) cp_async8(stasks + j, m.tile_tasks + tbeg + j);
      cp_async_commit();
      // halo element j: its 12 FP64 values staged by cp.async in the flux
      // region (unused until the edge phase) and converted to its FP32 slot
      // after the volume phase, so that the gather overlaps that phase
      const unsigned hst = smem_addr(res);
      for (int j = u; j < nh; j += kU) {
        const int g = m.tile_halo[hbeg + j];
        gid[j] = g;
        cp_async4(wds + kTile + j, A.wd + g);
#pragma unroll
        for (int r = 0; r < 9; ++r) cp_async8_s(hst + 96u * j + 8u * r, A.qin + (size_t)r * ne + g);
#pragma unroll
        for (int k = 0; k < 3; ++k) cp_async8_s(hst + 96u * j + 72u + 8u * k, m.hb + (size_t)k * ne + g);
      }
      cp_async_commit();
    }
    cp_async_wait_prior();
  }
  __syncthreads();
#else
  // Asynchronous global->shared copies (cp.async), no register staging, in
  // two groups: the tile's rows (state, bathymetry, geometry table, flags;
  // consecutive threads on consecutive elements of a row) and task words,
  // then the halo elements (thread j: halo element j's 13 values).  The
  // volume phase needs only the first group; the halo lands meanwhile.
  const int hg = tid < nh ? m.tile_halo[hbeg + tid] : -1;
  {
    // thread t: element t % kTile of every (kStageThreads / kTile)-th row;
    // shared addresses as 32-bit offsets, rows unrolled
    static_assert(kStageThreads % kTile == 0, "tile rows are copied by whole groups of kTile threads");
    constexpr int kRowStep = kStageThreads / kTile;
    const int w = tid % kTile, r0 = tid / kTile;
    const unsigned qs_s = smem_addr(qs), geo_s = smem_addr(geo);
    if (w < n) {
      const int ngeo = m.manning ? EGeo::kSmemRows : EGeo::kNbar;
      const size_t step = (size_t)kRowStep * ne;
      const unsigned qdst = qs_s + (unsigned)(w * kQStride + r0) * 8u;
      const double* src = A.qin + (size_t)r0 * ne + tile0 + w;
#pragma unroll
      for (int j = 0; j < (9 + kRowStep - 1) / kRowStep; ++j)
        if (r0 + j * kRowStep < 9) cp_async8_s(qdst + 8u * kRowStep * j, src + j * step);
      src = m.hb + (size_t)r0 * ne + tile0 + w;
#pragma unroll
      for (int j = 0; j < (3 + kRowStep - 1) / kRowStep; ++j)
        if (r0 + j * kRowStep < 3) cp_async8_s(qdst + 72u + 8u * kRowStep * j, src + j * step);
      constexpr unsigned rb = sizeof(real);
      const unsigned gdst = geo_s + (unsigned)(r0 * kTile + w) * rb;
      const real* gsrc = egeo_r(m) + (size_t)r0 * ne + tile0 + w;
#pragma unroll
      for (int j = 0; j < (EGeo::kSmemRows + kRowStep - 1) / kRowStep; ++j) {
        if (r0 + j * kRowStep >= ngeo) continue;
        if (rb == 8)
          cp_async8_s(gdst + rb * kRowStep * kTile * j, gsrc + j * step);
        else
          cp_async4_s(gdst + rb * kRowStep * kTile * j, gsrc + j * step);
      }
#pragma unroll
      for (int j = 0; j < (3 + kRowStep - 1) / kRowStep; ++j) {
        const int r = r0 + j * kRowStep;
        if (r == 0)
          cp_async4(wds + w, A.wd + tile0 + w);
        else if (r < 3)
          cp_async4(sinfo + (r - 1) * kTile + w, (r == 1 ? m.einfo : m.eslot) + tile0 + w);
      }
    }
    for (int j = tid; j < ntask; j += kStageThreads) cp_async8(stasks + j, m.tile_tasks + tbeg + j);
    cp_async_commit();
    for (int j = tid; j < nh; j += kStageThreads) {
      const int g = j == tid ? hg : m.tile_halo[hbeg + j];
      gid[j] = g;
      const unsigned hdst = qs_s + (unsigned)((kTile + j) * kQStride) * 8u;
      const double* q0 = A.qin + g;
#pragma unroll
      for (int c = 0; c < 9; ++c) cp_async8_s(hdst + 8u * c, q0 + (size_t)c * ne);
      const double* h0 = m.hb + g;
#pragma unroll
      for (int k = 0; k < 3; ++k) cp_async8_s(hdst + 72u + 8u * k, h0 + (size_t)k * ne);
      cp_async4(wds + kTile + j, A.wd + g);
    }
    cp_async_commit();
    // hybrid friction factor of tile element tid from the element-mean depth
    // (HB + ZE of mode 1, the operands the slot gets), for the volume phase
    if (P.iflinbf == 0 && P.ifhybf == 1 && tid < n) {
      const real depth_c = (real)(m.hb[tile0 + tid] + A.qin[tile0 + tid]);
      const real fh_c = real(1) / (kNonlin ? depth_c : real(P.nleq) * depth_c + real(P.leq));
      geo[SGeo::kHyb * kTile + tid] =
          pow(real(1) + pow(real(P.hbreak) * fh_c, real(P.ftheta)), real(P.fgamma / P.ftheta));
    }
    cp_async_wait_prior();
  }
  __syncthreads();
#endif

  // ---- phase 2: volume fluxes and sources per (element, area point) ----
  // (the point is the same for a whole warp: kTile is a multiple of 32)
  for (int w = tid; w < 3 * kTile; w += kStageThreads) {
    const int i = w / kTile, el = w - i * kTile;
    if (el >= n || wds[el] == 0) continue;
    volume_point<kNonlin, kSph, kTile>(A, cBasisR, qt, geo, vol, i, el, tile0 + el);
  }
  cp_async_wait_all();  // the halo group
#ifdef DGSWEM_MIXED
  for (int j = tid - kTile; j >= 0 && j < nh; j += kStageThreads - kTile) {
    const double* d = reinterpret_cast<const double*>(res) + 12 * j;  // this thread's staged copies
    float v[12];
#pragma unroll
    for (int r = 0; r < 9; ++r) v[r] = (float)d[r];
#pragma unroll
    for (int k = 0; k < 3; ++k) v[9 + k] = (float)(d[k] + d[9 + k]);
    float4* f = reinterpret_cast<float4*>(qt + (kTile + j) * kQfStride);
#pragma unroll
    for (int q = 0; q < 3; ++q) f[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
  }
#endif
  __syncthreads();

  // ---- phase 3: one thread per (edge task, Lobatto point) ----
  // (the three points of a task on adjacent lanes: same slots, broadcast loads)
  for (int w = tid; w < 3 * ntask; w += kStageThreads) {
    const int ti = w / 3, I = w - 3 * ti;
    const uint2 tk = stasks[ti];
    const unsigned fl = tk.x;
    const unsigned kind = fl & 7u;
    if (kind == kIBarrier) continue;  // ibarrier_sides, launched before this kernel
    real* o = res + (size_t)ti * 15 + 5 * I;
    const int sin = (fl >> TaskBits::kInSlot) & 511, sex = (fl >> TaskBits::kExSlot) & 511;
    const int led_in = (fl >> TaskBits::kLedIn) & 3, led_ex = (fl >> TaskBits::kLedEx) & 3;
    const bool flip = (fl >> TaskBits::kFlip) & 1u;
    const int owner = flip ? sex : sin, oled = flip ? led_ex : led_in;
    real nx = geo[(EGeo::kNx + oled) * kTile + owner], ny = geo[(EGeo::kNy + oled) * kTile + owner];
    if (flip) { nx = -nx; ny = -ny; }
    const int wd_in = wds[sin];
    // global ids for the ics=2 tables
    const int gin = sin < kTile ? tile0 + sin : gid[sin - kTile];
    if (kind == kInterior) {
      const int wd_ex = wds[sex];
      const int dry = wd_in == 0 && wd_ex == 0;
      if (I == 0) tdry[ti] = dry;
      if (dry) continue;
      const int gex = sex < kTile ? tile0 + sex : gid[sex - kTile];
      const int gp_in = I, gp_ex = 2 - I;
      real zi, xi, yi, wi, zx, xx, yx, wx, hi, hti, hx, htx;
      slot_trace(cBasisR, qt, sin, led_in, gp_in, zi, xi, yi, wi);
      slot_trace(cBasisR, qt, sex, led_ex, gp_ex, zx, xx, yx, wx);
      trace_depth<kNonlin>(P, zi, wi, hi, hti);
      trace_depth<kNonlin>(P, zx, wx, hx, htx);
      const real sfi = kSph ? (real)m.sfac_edge[(size_t)(led_in * 3 + gp_in) * ne + gin] : real(1);
      const real sfx = kSph ? (real)m.sfac_edge[(size_t)(led_ex * 3 + gp_ex) * ne + gex] : real(1);
      interior_point<kNonlin>(P, zi, zx, xi, xx, yi, yx, hi, hx, hti, htx, sfi, sfx, nx, ny, wd_in, wd_ex, o);
    } else {
      if (wd_in == 0) continue;
      real zi, xi, yi, wi, zx, xx, yx, hi, hti;
      slot_trace(cBasisR, qt, sin, led_in, I, zi, xi, yi, wi);
      trace_depth<kNonlin>(P, zi, wi, hi, hti);
      const real sfi = kSph ? (real)m.sfac_edge[(size_t)(led_in * 3 + I) * ne + gin] : real(1);
      ghost_state(A, kind, (int)tk.y, I, zi, xi, yi, hi, nx, ny, zx, xx, yx);
      // only the ocean ghost has its own elevation (the others copy zi)
      const real htx = kind == kOcean ? depth<kNonlin>(P, zx, hi) : hti;
      const Flux3T<real> f =
          llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hi, hti, htx, sfi, sfi, nx, ny, real(P.g));
      o[0] = f.f; o[1] = f.g; o[2] = f.h;
    }
  }
  __syncthreads();


  // ---- phase 4: per (element, mode) sums in the reference's order, SSP ----
  for (int w = tid; w < 3 * kTile; w += kStageThreads) {
    const int K = w / kTile, el = w - K * kTile;
    if (el >= n) continue;
    sum_mode<kNonlin, kTile>(A, qs, geo, vol, res, tdry, sinfo, wds, stasks, K, el, tile0 + el);
  }
}

// slopelimiter.F:3300-3404: min/max of element means over each node's star,
// stored as (min, max) pairs per variable, minmax[(var*NP + n)*2 + {0,1}]:
// the limiter pass gathers a node's bounds of a variable with one 16-byte
// load (one sector; six separate arrays took two 8-byte loads from two
// sectors), and this pass writes three coalesced pair arrays.
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
  const size_t np = (size_t)L.m.np;
  double2* o = reinterpret_cast<double2*>(L.minmax);
  o[n] = make_double2(zmin, zmax);
  o[np + n] = make_double2(xmin, xmax);
  o[2 * np + n] = make_double2(ymin, ymax);
}

// bounds (min, max) of variable var at node nd
__device__ __forceinline__ double2 node_bounds(const double* minmax, int np, int nd, int var) {
  return reinterpret_cast<const double2*>(minmax)[(size_t)var * np + nd];
}

// x / 3 in the arithmetic type: the correctly rounded FP64 quotient without
// a division (div3, cr_math.cuh), the FP32 division in the mixed variant
__device__ __forceinline__ double third_of(double x) { return div3(x); }
__device__ __forceinline__ float third_of(float x) { return x / 3.0f; }

// x / d for the redistribution divisor d = max(1, kdp) in {1, 2, 3}: x / 1
// and x / 2 are exact scalings (x * 0.5 is the same correctly rounded value
// as x / 2), x / 3 the correctly rounded quotient.
__device__ __forceinline__ real div_count(real x, int kdp) {
  if (kdp <= 1) return x;
  if (kdp == 2) return x * real(0.5);
  return third_of(x);
}

// slopelimiter.F:3434-3779 (vertex clamp + 3 redistribution sweeps) followed
// by wetdry.F:61-548 for the same element.  The limiter arithmetic is in the
// arithmetic type (FP32 in the mixed variant, on deviations from the element
// mean, which it does not change), WETDRY in FP64.
// Compiled per limiter shape (kLimitBlocks / kLimitMinBlocks): 1024 resident
// threads per SM (64 registers, no spills: more warps to cover the
// limiter's dependent FP64 chains than an unbounded allocation allows) in
// blocks of 256 or 128, or 768 (85 registers).
template <int kBlock, int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks) limit_wetdry(const __grid_constant__ LimitArgs L) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = L.m.ne, np = L.m.np;
  if (e >= L.ne_act) return;
  const BasisP1& B = cBasis;
  int nd[3];
#pragma unroll
  for (int v = 0; v < 3; ++v) nd[v] = L.m.nm[(size_t)v * ne + e];
  double q[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) q[c] = L.q[(size_t)c * ne + e];
  // the element means (mode 1 of ZE, QX, QY) and WDFLG change only in
  // WETDRY: values whose bits did not change are not stored again (modes
  // 2-3 are rebuilt by the limiter and stored always)
  const double m0 = q[0], m3 = q[3], m6 = q[6];
#ifdef DGSWEM_MIXED
  // mixed variant: modes 2-3 of a variable are stored only where the
  // limiter rebuilt them or WETDRY changed a mode
  bool rebuilt[3] = {false, false, false}, wd_modes = false;
#endif
  if (L.slopeflag != 0) {
#pragma unroll
    for (int var = 0; var < 3; ++var) {
      double* zc = &q[3 * var];
#ifdef DGSWEM_MIXED
      // FP32 on deviations from the element mean (mode 1): vertex value -
      // mode 1 and bound - mode 1 (differences in FP64).  The sweeps and
      // the rebuild of modes 2-3 are the reference's with mode 1 = 0 (the
      // mean cancels exactly in both), so FP32 rounds only the small
      // deviations, not the full vertex values.  A variable whose three
      // vertex values lie within their bounds is left as it is: the clamp
      // changes nothing, and the sweeps and the rebuild are the identity in
      // exact arithmetic (the reference's FP64 rebuild returns the modes to
      // rounding), so its FP64 modes are kept rather than rounded to FP32.
      const real z0 = 0;
      real vmin[3], vmax[3], vx[3];
      bool clamped = false;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double2 bd = node_bounds(L.minmax, np, nd[a], var);
        vmin[a] = (real)(bd.x - zc[0]);
        vmax[a] = (real)(bd.y - zc[0]);
        const real v = (real)(B.phi_corner[a][1] * zc[1] + B.phi_corner[a][2] * zc[2]);
        vx[a] = fmax(fmin(v, vmax[a]), vmin[a]);
        clamped = clamped || v > vmax[a] || v < vmin[a];
      }
      if (!clamped) continue;
      rebuilt[var] = true;
#else
      const real z0 = zc[0];
      real vmin[3], vmax[3], vx[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double2 bd = node_bounds(L.minmax, np, nd[a], var);
        vmin[a] = bd.x;
        vmax[a] = bd.y;
        vx[a] = zc[0] + B.phi_corner[a][1] * zc[1] + B.phi_corner[a][2] * zc[2];
        vx[a] = fmax(fmin(vx[a], vmax[a]), vmin[a]);
      }
#endif
#pragma unroll
      for (int sweep = 0; sweep < 3; ++sweep) {
        const real sumloc = third_of(vx[0] + vx[1] + vx[2]);
        real sumdif = (sumloc - z0) * real(3);
        // A sweep that starts from sumdif == +0 with every vx - vmin free of
        // a sign bit changes no bit: each redfac is +0 (the quotient of +0,
        // or 0, capped by a non-negative redmax), so vx - redfac leaves vx
        // (a -0 included) and the next sweep starts from the same values.
        // Stopping there gives the bits of running all three sweeps.
        if (!signbit(sumdif) && sumdif == real(0) && !signbit(vx[0] - vmin[0]) && !signbit(vx[1] - vmin[1]) &&
            !signbit(vx[2] - vmin[2]))
          break;
        const real signdif = copysign(real(1), sumdif);
        real dif[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) dif[a] = (vx[a] - z0) * signdif;
        int kdp = (dif[0] > 0) + (dif[1] > 0) + (dif[2] > 0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          real redfac = 0;
          if (dif[k] > 0) {  // sumdif * signdif / max(1, kdp)
            redfac = div_count(sumdif * signdif, kdp);
            kdp = kdp - 1;
          }
          const real redmax = signdif > 0 ? vx[k] - vmin[k] : vmax[k] - vx[k];
          redfac = fmin(redfac, redmax);
          sumdif = sumdif - redfac * signdif;
          vx[k] = vx[k] - redfac * signdif;
        }
      }
      zc[1] = -(real(1.0 / 6.0) * (vx[0] + vx[1])) + real(1.0 / 3.0) * vx[2];
      zc[2] = -(real(.5) * vx[0]) + real(.5) * vx[1];
    }
  }
  if (L.wetdry) {
    const double H0 = L.ph.h0, ZERO = 1.0e-6, c13 = 1.0 / 3.0, c16 = 1.0 / 6.0;
    double dpn[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) dpn[v] = L.m.dp[nd[v]];
    const double dpe_min = fmin(fmin(dpn[0], dpn[1]), dpn[2]);
    int wd = L.wd[e];
    const int wd_read = wd;
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
#ifdef DGSWEM_MIXED
      wd_modes = true;
#endif
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
        // vertices shallow -> deep: the reference's exchange sort of the
        // index list (pairs (1,2), (1,3), (2,3) in that order, swapping when
        // the first depth is larger), held as (depth, vertex) registers
        double s0 = ht[0], s1 = ht[1], s2 = ht[2];
        int j0 = 0, j1 = 1, j2 = 2;
        if (s0 > s1) { const double t = s0; s0 = s1; s1 = t; const int u = j0; j0 = j1; j1 = u; }
        if (s0 > s2) { const double t = s0; s0 = s2; s2 = t; const int u = j0; j0 = j2; j2 = u; }
        if (s1 > s2) { const double t = s1; s1 = s2; s2 = t; const int u = j1; j1 = j2; j2 = u; }
        const double d0 = fmax(H0, s0) - s0;
        const double d1 = fmax(H0, s1 - 0.5 * d0) - s1;
        const double d2 = -d0 - d1;
        double dh[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) dh[v] = j0 == v ? d0 : (j1 == v ? d1 : d2);
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
          // / (3 - nd2), nd2 in {0, 1, 2}: by 3 correctly rounded, by 2 and 1 exact
          qxs = nd2 == 0 ? div3(qxs) : nd2 == 1 ? qxs * 0.5 : qxs;
          qys = nd2 == 0 ? div3(qys) : nd2 == 1 ? qys * 0.5 : qys;
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
      const double zmax = hmax_i == 0 ? zh[0] : (hmax_i == 1 ? zh[1] : zh[2]);
      if (zmax > (-dpe_min + H0)) {
        wd = 1;
      } else {
#pragma unroll
        for (int c = 3; c < 9; ++c) q[c] = 0.0;
        wd = 0;
#ifdef DGSWEM_MIXED
        wd_modes = true;
#endif
      }
    }
    if (wd != wd_read) L.wd[e] = wd;
  }
  auto same = [](double a, double b) { return __double_as_longlong(a) == __double_as_longlong(b); };
  if (!same(q[0], m0)) L.q[e] = q[0];
  if (!same(q[3], m3)) L.q[(size_t)3 * ne + e] = q[3];
  if (!same(q[6], m6)) L.q[(size_t)6 * ne + e] = q[6];
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    if (c % 3 == 0) continue;
#ifdef DGSWEM_MIXED
    if (!rebuilt[c / 3] && !wd_modes) continue;
#endif
    L.q[(size_t)c * ne + e] = q[c];
  }
}

// write_results.F:14-170 (modal2nodal) + NODECODE from the wet flags; node n
// of the device order writes its results at its input position
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
  const int out = m.node_perm[n];  // results in the input node order
  if (eta2) eta2[out] = et;
  if (uu2) uu2[out] = uu;
  if (vv2) vv2[out] = vv;
  if (nodecode) nodecode[out] = wet;
}

// Fortran layout ZE(DOFH,NE) <-> state SoA q[c*NE+e] for one variable
// Host (Fortran) layout f[3*e + k] in input element order <-> device SoA
// q[(3*var + k)*NE + i] in device element order: i = inv[e], e = perm[i].
__global__ void fortran_to_soa(const double* __restrict__ f, double* __restrict__ q, int ne, int var,
                               const int* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const int e = perm[i];
#pragma unroll
  for (int k = 0; k < 3; ++k) q[(size_t)(3 * var + k) * ne + i] = f[(size_t)3 * e + k];
}

__global__ void soa_to_fortran(const double* __restrict__ q, double* __restrict__ f, int ne, int var,
                               const int* __restrict__ inv) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int i = inv[e];
#pragma unroll
  for (int k = 0; k < 3; ++k) f[(size_t)3 * e + k] = q[(size_t)(3 * var + k) * ne + i];
}

// Halo of a partitioned handle: the states of stage buffer q (row stride ne)
// at local element ids idx[0..n) to / from a contiguous buffer.  kind 0: the
// element means of ZE, QX, QY (3 doubles); kind 1: the nine modal values and
// WDFLG (10 doubles, WDFLG as 0.0 / 1.0).
__global__ void halo_pack(const double* __restrict__ q, const int* __restrict__ wd, int ne,
                          const int* __restrict__ idx, int n, int kind, double* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = idx[j];
  if (kind == 0) {
#pragma unroll
    for (int v = 0; v < 3; ++v) out[(size_t)3 * j + v] = q[(size_t)(3 * v) * ne + i];
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) out[(size_t)10 * j + c] = q[(size_t)c * ne + i];
    out[(size_t)10 * j + 9] = (double)wd[i];
  }
}

__global__ void halo_unpack(double* __restrict__ q, int* __restrict__ wd, int ne, const int* __restrict__ idx,
                            int n, int kind, const double* __restrict__ in) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = idx[j];
  if (kind == 0) {
#pragma unroll
    for (int v = 0; v < 3; ++v) q[(size_t)(3 * v) * ne + i] = in[(size_t)3 * j + v];
  } else {
#pragma unroll
    for (int c = 0; c < 9; ++c) q[(size_t)c * ne + i] = in[(size_t)10 * j + c];
    wd[i] = (int)in[(size_t)10 * j + 9];
  }
}

// dst[i] = src[idx[i]]: WDFLG between input and device element order
__global__ void gather_int(const int* __restrict__ src, int* __restrict__ dst, const int* __restrict__ idx, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

}  // namespace DGSWEM_VARIANT
}  // namespace dgswem
