// hydro_p2.cuh -- the p=2 stage (six modes per variable, four Gauss-Lobatto
// points per edge, the six-point area rule): a tile kernel per RK stage, or
// an edge kernel and an element kernel where a tile does not fit shared
// memory.  Included after hydro_kernels.cuh (its LLF flux, depth,
// trace_depth, the arithmetic type `real`) by kernels_p2_fast.cu /
// kernels_p2_strict.cu (FP64) and kernels_p2_mixed.cu (edge traces, fluxes
// and volume terms in FP32; the right-hand-side sums and their weights, the
// state, the SSP combination and the ocean depth-positivity fix in FP64)
// with DGSWEM_VARIANT set.
// The arithmetic follows the p=1 kernels term for term, generalised over the
// modes and points as the reference's p-generic boundary-edge code
// (land_edge_hydro.F:144,273) is; the interior-edge sums run over every mode
// (the reference's internal_edge_hydro.F:306-318 sums modes 1-3 only, its
// p=2 defect).  No wetting/drying and no slope limiter at p=2 (both are p=1
// only in the reference); land, ocean and interior edges; ICS=1.
#pragma once

namespace dgswem {
namespace DGSWEM_VARIANT {

__constant__ BasisP2 cB2;
__constant__ BasisP2T<real> cB2R;  // cB2 in the arithmetic type

// The fourth modal row of element e in the arithmetic type: the bathymetry
// mode HB_k (FP64 variants) or the depth mode ZE_k + HB_k summed in FP64 and
// rounded (mixed), as the p=1 kernels' slots.
__device__ __forceinline__ real fourth_mode(const double* __restrict__ q, const double* __restrict__ hb, int ne,
                                            int e, int k) {
#ifdef DGSWEM_MIXED
  return (real)(q[(size_t)k * ne + e] + hb[(size_t)k * ne + e]);
#else
  return hb[(size_t)k * ne + e];
#endif
}

// Traces of ZE, QX, QY and the fourth row (HB, or the depth in the mixed
// variant; see trace_depth) at one point from the six modes (state rows
// 6*var + k, bathymetry rows k), summed from mode 1 upwards as the
// reference's trace loops are (mode 1 is 1 at every point).
__device__ __forceinline__ void trace6(const double* __restrict__ q, const double* __restrict__ hb, int ne,
                                       int e, const real* phi, real& z, real& u, real& v, real& h) {
  z = (real)q[e];
  u = (real)q[(size_t)6 * ne + e];
  v = (real)q[(size_t)12 * ne + e];
  h = fourth_mode(q, hb, ne, e, 0);
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) {
    z = z + (real)q[(size_t)k * ne + e] * phi[k];
    u = u + (real)q[(size_t)(6 + k) * ne + e] * phi[k];
    v = v + (real)q[(size_t)(12 + k) * ne + e] * phi[k];
    h = h + fourth_mode(q, hb, ne, e, k) * phi[k];
  }
}

// Edge part: one thread per (edge of A.edges, Lobatto point): interior edges
// once, from their in side NEDEL(1) in the reference's orientation, and land
// and ocean edges.  The LLF flux (F, G, H) at the point goes to both sides'
// slots ef[((e*3 + led)*4 + point)*3 + c], each side at its own point index
// (the ex side's point order is reversed), one writer per slot.
// internal_edge_hydro.F, land_edge_hydro.F, ocean_edge_hydro.F
template <bool kNonlin>
__global__ void __launch_bounds__(128) p2_edges(const __grid_constant__ P2Args A) {
  const long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= (long long)kP2Egp * A.nedge) return;
  const int ed = (int)(w / kP2Egp), I = (int)(w - (long long)ed * kP2Egp);
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const BasisP2T<real>& B = cB2R;
  const int ne = m.ne;
  const int e = A.edges[2 * ed], l = A.edges[2 * ed + 1];
  const unsigned info = m.einfo[e], kind = ei_kind(info, l);
  const real* G = egeo_r(m);
  const real nx = G[(size_t)(EGeo::kNx + l) * ne + e], ny = G[(size_t)(EGeo::kNy + l) * ne + e];
  real* ef = reinterpret_cast<real*>(A.ef);
  real zi, xi, yi, wi, hi, hti;
  trace6(A.qin, m.hb, ne, e, B.phi_edge[l][I], zi, xi, yi, wi);
  trace_depth<kNonlin>(P, zi, wi, hi, hti);
  real* o = ef + ((size_t)(e * 3 + l) * kP2Egp + I) * 3;
  if (kind == kInterior) {
    const int ex = m.link[(size_t)l * ne + e], lx = (int)ei_nled(info, l), J = kP2Egp - 1 - I;
    real zx, xx, yx, wx, hx, htx;
    trace6(A.qin, m.hb, ne, ex, B.phi_edge[lx][J], zx, xx, yx, wx);
    trace_depth<kNonlin>(P, zx, wx, hx, htx);
    const Flux3T<real> f =
        llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hx, hti, htx, real(1), real(1), nx, ny, real(P.g));
    o[0] = f.f; o[1] = f.g; o[2] = f.h;
    real* ox = ef + ((size_t)(ex * 3 + lx) * kP2Egp + J) * 3;
    ox[0] = f.f; ox[1] = f.g; ox[2] = f.h;
    return;
  }
  // ghost state: land reflects the normal momentum (land_edge_hydro.F:201-218);
  // ocean takes the harmonic elevation with the depth-positivity fix
  // (ocean_edge_hydro.F:148-177, 255-259; FP64 in every variant) and the
  // interior momentum
  real zx = zi, xx = xi, yx = yi, htx = hti;
  if (kind == kOcean) {
    const int list = m.link[(size_t)l * ne + e];
    double zsum = 0.0;
    for (int f = 0; f < m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * cB2.xegp[I]);
    }
    const double hid = hi;
    if (zsum * P.ifnlfa + hid <= 0) zsum = fabs(hid) + P.h0;
    zx = (real)zsum;
    htx = depth<kNonlin>(P, zx, hi);
  } else {
    const real tx = -ny, ty = nx;
    const real qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const real qne = -qn, qte = qt, den = real(1) / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  }
  const Flux3T<real> f =
      llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hi, hti, htx, real(1), real(1), nx, ny, real(P.g));
  o[0] = f.f; o[1] = f.g; o[2] = f.h;
}


// Physics constants in the arithmetic type
__device__ __forceinline__ PhysR phys_r(const P2Args& A) {
#ifdef DGSWEM_MIXED
  const PhysF& p = A.pf;
#else
  const Physics& p = A.ph;
#endif
  return PhysR{p.g, p.nleq, p.leq, p.nleqg, p.fg_l, p.tau_cap, p.cori, p.fric, p.cf};
}

// Volume fluxes and sources at area point i of element e (rhs_dg_hydro.F:58-470
// with six modes): out = fx fy gx gy hx hy sx sy.  q: the element's 18 state
// values (row 6*var + k) and w its six fourth-row modes (fourth_mode: HB, or
// the depth modes in the mixed variant), in the arithmetic type.
// Per-element terms of the volume integral, in the arithmetic type: the
// Coriolis parameter and the bottom friction coefficient (nodal arrays or the
// constants), Manning's n, and the vertices' wind stress and pressure scaled
// by the stage's ramp (met_forcing.F:49-66).
struct P2Frc {
  real cori, fric, nbar, wx[3], wy[3], pr[3];
  // rows a tile keeps in shared memory: all but nbar (a geometry row)
  static constexpr int kRows = 11;
};
__device__ __forceinline__ P2Frc p2_force(const P2Args& A, int e) {
  const MeshView& m = A.m;
  const PhysR R = phys_r(A);
  const int ne = m.ne;
  P2Frc F;
  F.cori = m.cori ? (real)m.cori[e] : R.cori;
  F.fric = m.fric ? (real)m.fric[e] : R.fric;
  F.nbar = m.manning ? egeo_r(m)[(size_t)EGeo::kNbar * ne + e] : real(0);
  if (A.ph.nws != 0) {
    const real r = (real)(A.ramp ? *A.ramp : A.rampdg);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int n = m.nm[(size_t)a * ne + e];
      F.wx[a] = r * (real)A.wsx[n];
      F.wy[a] = r * (real)A.wsy[n];
      F.pr[a] = r * (real)A.pr[n];
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) F.wx[a] = F.wy[a] = F.pr[a] = real(0);
  }
  return F;
}

template <bool kNonlin>
__device__ __forceinline__ void p2_volume(const P2Args& A, const real* q, const real* w, real drdx, real dsdx,
                                          real drdy, real dsdy, real hyb, const P2Frc& F, int i, real out[8]) {
  const Physics& P = A.ph;
  const PhysR R = phys_r(A);
  const BasisP2T<real>& C = cB2R;
#ifdef DGSWEM_MIXED
  real hbe[kP2Modes];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) hbe[k] = w[k] - q[k];
#else
  const real* hbe = w;
#endif
  const real NLEQ = kNonlin ? real(1) : R.nleq, LEQ = kNonlin ? real(0) : R.leq;
  const real cori = F.cori;
  real fric = F.fric;
  real zq = q[0], uq = q[6], vq = q[12];
  real hq = hbe[0] * C.phi_area[0][i];
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) hq = hq + hbe[k] * C.phi_area[k][i];
  real dhx = 0, dhy = 0;
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) {
    dhx = dhx + hbe[k] * (C.drphi[k][i] * drdx + C.dsphi[k][i] * dsdx);
    dhy = dhy + hbe[k] * (C.drphi[k][i] * drdy + C.dsphi[k][i] * dsdy);
  }
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) {
    zq = zq + q[k] * C.phi_area[k][i];
    uq = uq + q[6 + k] * C.phi_area[k][i];
    vq = vq + q[12 + k] * C.phi_area[k][i];
  }
#ifdef DGSWEM_MIXED
  // the depth from the depth modes (a thin column keeps FP32 relative accuracy)
  real depth = w[0] * C.phi_area[0][i];
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) depth = depth + w[k] * C.phi_area[k][i];
  if (!kNonlin) depth = zq + hq;
#else
  const real depth = zq + hq;
#endif
  const real f1 = kNonlin ? real(1) : NLEQ + LEQ * hq;
  const real fx = uq * f1 * real(1), fy = vq * f1;
  const real fu = kNonlin ? uq : NLEQ * uq, fv = kNonlin ? vq : NLEQ * vq;
  const real fg = R.nleqg * zq * 1;
  const real fh = real(1) / (kNonlin ? depth : NLEQ * depth + LEQ);
  const real u = uq * fh, v = vq * fh;
  const real huu = fu * u, hvv = fv * v, huv = fu * v;
  const real gh2 = kNonlin ? fg * (real(0.5) * zq + hq) : fg * (real(0.5) * zq + hq) + R.fg_l * zq;
  const real gx = (huu + gh2) * real(1), gy = huv;
  const real hx = huv * real(1), hy = hvv + gh2;
  if (A.m.manning) {
    const real nbar = F.nbar;
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
  real sx = -(tau * uq) + fg * dhx * real(1) + cori * vq;
  real sy = -(tau * vq) + fg * dhy - cori * uq;
  if (P.nws != 0) {
    // met_forcing.F:49-66: the nodal fields scaled by the stage's ramp
    const real drpsi[3] = {-0.5, 0.5, 0.0}, dspsi[3] = {-0.5, 0.0, 0.5};
    real dpsidx[3], dpsidy[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dpsidx[a] = drpsi[a] * drdx + dspsi[a] * dsdx;
      dpsidy[a] = drpsi[a] * drdy + dspsi[a] * dsdy;
    }
    const real fw = real(1) / f1;
    sx = sx + fw * (F.wx[0] * C.psi[0][i] + F.wx[1] * C.psi[1][i] + F.wx[2] * C.psi[2][i]) -
         R.g * real(1) * depth * (F.pr[0] * dpsidx[0] + F.pr[1] * dpsidx[1] + F.pr[2] * dpsidx[2]);
    sy = sy + fw * (F.wy[0] * C.psi[0][i] + F.wy[1] * C.psi[1][i] + F.wy[2] * C.psi[2][i]) -
         R.g * depth * (F.pr[0] * dpsidy[0] + F.pr[1] * dpsidy[1] + F.pr[2] * dpsidy[2]);
  }
  out[0] = fx; out[1] = fy; out[2] = gx; out[3] = gy;
  out[4] = hx; out[5] = hy; out[6] = sx; out[7] = sy;
}

// Element part: one thread per owned element.  Per variable the six modes'
// right-hand side in the reference's order -- boundary edges by kind and
// list, interior edges as the slot sum of add_internal_flux, rain, area
// points -- then the SSP combination (DG_hydro_timestep.F:238-290) into
// qout.  Every element is wet at p=2.  The three variables' sums are
// accumulated together, each in that order, the volume terms of an area
// point used as soon as they are formed.  Compiled for four resident
// blocks of 128 per SM (128 registers, about 500 bytes of spills to
// L1-cached local memory): latency bound, it gains more from the warps than
// it loses to the spills (8M-element step: 9.48 ms; three blocks, 168
// registers: 10.20 ms; two blocks, 247 registers: 9.75 ms).
template <bool kNonlin>
__global__ void __launch_bounds__(128, 4) p2_elements(const __grid_constant__ P2Args A) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= A.ne_act) return;
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const BasisP2T<real>& B = cB2R;
  const int ne = m.ne;
  const real* G = egeo_r(m);
  const real* ef = reinterpret_cast<const real*>(A.ef);
  real q[3 * kP2Modes], wm[kP2Modes];
#pragma unroll
  for (int c = 0; c < 3 * kP2Modes; ++c) q[c] = (real)A.qin[(size_t)c * ne + e];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) wm[k] = fourth_mode(A.qin, m.hb, ne, e, k);
  const real drdx = G[(size_t)EGeo::kDrdx * ne + e], dsdx = G[(size_t)EGeo::kDsdx * ne + e];
  const real drdy = G[(size_t)EGeo::kDrdy * ne + e], dsdy = G[(size_t)EGeo::kDsdy * ne + e];
  real hyb = 1;
  if (P.iflinbf == 0 && P.ifhybf == 1) {
#ifdef DGSWEM_MIXED
    const real depth_c = wm[0];  // depth mode 1
#else
    const real depth_c = wm[0] + q[0];
#endif
    const real fh_c = real(1) / (kNonlin ? depth_c : real(P.nleq) * depth_c + real(P.leq));
    hyb = pow(real(1) + pow(real(P.hbreak) * fh_c, real(P.ftheta)), real(P.fgamma / P.ftheta));
  }
  // all three variables' sums at once (no per-point volume array): each
  // (variable, mode) sum takes the same terms in the same order as above
  // (the sums and their weights in FP64 in every variant, as p2_tile's)
#ifdef DGSWEM_MIXED
  using acc_t = double;
  const BasisP2& W = cB2;
  const acc_t drdxw = drdx, dsdxw = dsdx, drdyw = drdy, dsdyw = dsdy;
#else
  using acc_t = real;
  const BasisP2T<real>& W = B;
  const real drdxw = drdx, dsdxw = dsdx, drdyw = drdy, dsdyw = dsdy;
#endif
  const unsigned info = m.einfo[e];
  acc_t rhs[3][kP2Modes], isum[3][kP2Modes];
#pragma unroll
  for (int V = 0; V < 3; ++V)
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) { rhs[V][k] = 0; isum[V][k] = 0; }
  for (int s = 0; s < 3; ++s) {
    const int l = ei_order(info, s);
    const unsigned kind = ei_kind(info, l);
    if (kind == kNone) continue;
    const real* efl = ef + (size_t)(e * 3 + l) * kP2Egp * 3;
    if (kind == kInterior) {
      const bool is_in = ei_flag(info, l) != 0;
      const acc_t edfac = G[(size_t)(EGeo::kEdfac + l) * ne + e];
      acc_t acc[3][kP2Modes];
#pragma unroll
      for (int V = 0; V < 3; ++V)
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) acc[V][k] = 0;
      for (int I = 0; I < kP2Egp; ++I) {
        const int j = is_in ? I : kP2Egp - 1 - I;
        const acc_t v0 = efl[j * 3], v1 = efl[j * 3 + 1], v2 = efl[j * 3 + 2];
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) {
          const acc_t wk = edfac * W.edgeq[l][j][k];
          if (is_in) {
            acc[0][k] = acc[0][k] - wk * v0;
            acc[1][k] = acc[1][k] - wk * v1;
            acc[2][k] = acc[2][k] - wk * v2;
          } else {
            acc[0][k] = acc[0][k] + wk * v0;
            acc[1][k] = acc[1][k] + wk * v1;
            acc[2][k] = acc[2][k] + wk * v2;
          }
        }
      }
#pragma unroll
      for (int V = 0; V < 3; ++V)
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) isum[V][k] = isum[V][k] + acc[V][k];
    } else {
      const acc_t areas = G[(size_t)EGeo::kAreas * ne + e];
      const acc_t xlen = G[(size_t)(EGeo::kXlen + l) * ne + e];
      for (int I = 0; I < kP2Egp; ++I) {
        const acc_t v0 = efl[I * 3], v1 = efl[I * 3 + 1], v2 = efl[I * 3 + 2];
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) {
          const acc_t wk = acc_t(2) * W.m_inv[k] / areas * xlen * W.phi_edge[l][I][k] * W.wegp[I];
          rhs[0][k] = rhs[0][k] - wk * v0;
          rhs[1][k] = rhs[1][k] - wk * v1;
          rhs[2][k] = rhs[2][k] - wk * v2;
        }
      }
    }
  }
#pragma unroll
  for (int V = 0; V < 3; ++V)
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) rhs[V][k] = rhs[V][k] + isum[V][k];  // add_internal_flux
  if (P.rainfall == 1) {
    const acc_t src = acc_t(7.0556e-6);
    for (int i = 0; i < kP2Agp; ++i)
#pragma unroll
      for (int k = 0; k < kP2Modes; ++k) rhs[0][k] = rhs[0][k] + W.srfac[k][i] * src;
  }
  for (int i = 0; i < kP2Agp; ++i) {
    real vol[8];
    p2_volume<kNonlin>(A, q, wm, drdx, dsdx, drdy, dsdy, hyb, p2_force(A, e), i, vol);
    acc_t vw[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) vw[r] = vol[r];
    rhs[1][0] = rhs[1][0] + W.srfac[0][i] * vw[6];
    rhs[2][0] = rhs[2][0] + W.srfac[0][i] * vw[7];
#pragma unroll
    for (int k = 1; k < kP2Modes; ++k) {
      const acc_t dpx = W.drphi[k][i] * drdxw + W.dsphi[k][i] * dsdxw;
      const acc_t dpy = W.drphi[k][i] * drdyw + W.dsphi[k][i] * dsdyw;
      const acc_t xf = W.mw[k][i] * dpx;
      const acc_t yf = W.mw[k][i] * dpy;
      const acc_t sr = W.srfac[k][i];
      rhs[0][k] = rhs[0][k] + xf * vw[0] + yf * vw[1];
      rhs[1][k] = rhs[1][k] + xf * vw[2] + yf * vw[3] + sr * vw[6];
      rhs[2][k] = rhs[2][k] + xf * vw[4] + yf * vw[5] + sr * vw[7];
    }
  }
  // SSP-RK combination (DG_hydro_timestep.F:238-290) in FP64; zero
  // coefficients skipped
  bool bad = false;
  const bool hist0 = A.irk > 1;
#pragma unroll
  for (int V = 0; V < 3; ++V)
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) {
      const int c = kP2Modes * V + k;
      const double rk = (double)rhs[V][k];
      if (A.rout) A.rout[(size_t)c * ne + e] = rk;
      const double qc = A.qin[(size_t)c * ne + e];
      double acc = 0.0;
      if (hist0) {
        if (A.a[0] != 0.0) acc = acc + A.a[0] * A.qhist[0][(size_t)c * ne + e];
        if (A.b[0] != 0.0) acc = acc + A.b[0] * A.rhist[0][(size_t)c * ne + e];
      }
      for (int I = 1; I < A.irk; ++I) {
        const bool cur = I == A.irk - 1;
        if (A.a[I] != 0.0) acc = acc + A.a[I] * (cur ? qc : A.qhist[I][(size_t)c * ne + e]);
        if (A.b[I] != 0.0) acc = acc + A.b[I] * (cur ? rk : A.rhist[I][(size_t)c * ne + e]);
      }
      if (!hist0) {
        if (A.a[0] != 0.0) acc = acc + A.a[0] * qc;
        if (A.b[0] != 0.0) acc = acc + A.b[0] * rk;
      }
      bad = bad || isnan(acc);
      A.qout[(size_t)c * ne + e] = acc;
    }
  if (bad) atomicOr(A.err, 1u);
}

// ---------------------------------------------------------------------------
// p=2 tile kernel: the p=1 tile kernel's scheme at six modes.  Block b owns
// tile b of the tile plan (consecutive elements of the Morton order, their
// edge tasks, the out-of-tile neighbours those read), phases separated by
// barriers:
//   1. tile and halo elements' 24 slot values (18 modal values, six fourth-
//      row modes: HB, or the depth modes in the mixed variant), the tile's
//      geometry rows, edge info, task words and per-element forcing terms
//      (P2Frc: Coriolis, friction, the vertices' wind and pressure) into
//      shared memory, and the hybrid friction factor of each tile element;
//   2. one work item per thread and round over the tile's edge points and
//      then its area points: an edge point (edge task, Lobatto point) gives
//      the LLF flux of the point in the reference's in/ex orientation, or the
//      land / ocean ghost and its flux -> (F, G, H); an area point (element,
//      point) gives its volume fluxes and sources;
//   3. one thread per (element, mode): the mode's right-hand side of the
//      three variables in the order of p2_elements (boundary edges, interior
//      edges as the slot sum, rain, area points), then the SSP combination,
//      its state operands loaded before the sums.
// Each interior edge point is evaluated once per tile (twice for an edge
// between tiles) and its flux stays in shared memory: no flux slots in HBM.
// Every sum has p2_elements' operands and order, so both give the same bits.
// internal_edge_hydro.F, land_edge_hydro.F, ocean_edge_hydro.F,
// rhs_dg_hydro.F, DG_hydro_timestep.F:238-290
// ---------------------------------------------------------------------------
constexpr int kP2Tile = 64, kP2TileThreads = 384;
// slot stride in reals: 24 values and a pad keeping 16-byte loads by
// consecutive slots off one bank group (13 or 7 16-byte units, odd)
constexpr int kP2SlotStride = sizeof(real) == 8 ? 26 : 28;
constexpr int kP2Vol = 8;  // fx fy gx gy hx hy sx sy
// reals per edge task's flux slots (four points x F, G, H and a pad): an odd
// stride spreads the tasks that a warp's elements read over the banks
constexpr int kP2ResStride = 3 * kP2Egp + 1;

// the edge traces' basis values, read with per-lane indices (local edge and
// point vary across a warp) by the edge points, kept in shared memory with
// rows of seven (the twelve (edge, point) rows a warp reads fall on
// distinct banks); the sums read their edge weights from constant memory,
// which takes that load off the shared-memory pipe
constexpr int kP2EbRow = kP2Modes + 1;
struct P2EdgeBasis {
  real phi_edge[3][kP2Egp][kP2EbRow];
};

struct P2Layout {
  unsigned qs, geo, frc, vol, res, info, tasks, bytes;
};
__host__ __device__ inline P2Layout p2_layout(int max_halo, int max_tasks) {
  P2Layout L;
  const unsigned S = (unsigned)(kP2Tile + max_halo), T = (unsigned)max_tasks, rb = (unsigned)sizeof(real);
  L.qs = align16((unsigned)sizeof(P2EdgeBasis));
  L.geo = align16(L.qs + S * kP2SlotStride * rb);
  L.frc = align16(L.geo + kGeoRows * kP2Tile * rb);
  L.vol = align16(L.frc + P2Frc::kRows * kP2Tile * rb);
  L.res = align16(L.vol + kP2Vol * kP2Agp * kP2Tile * rb);
  L.info = align16(L.res + T * kP2ResStride * rb);
  L.tasks = align16(L.info + 2u * kP2Tile * 4u);
  L.bytes = align16(L.tasks + T * 8u);
  return L;
}

// the 24 slot values of element g (device id) from global memory
__device__ __forceinline__ void p2_slot_store(const P2Args& A, int g, real* dst) {
  const int ne = A.m.ne;
#pragma unroll
  for (int c = 0; c < 3 * kP2Modes; ++c) dst[c] = (real)A.qin[(size_t)c * ne + g];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) dst[3 * kP2Modes + k] = fourth_mode(A.qin, A.m.hb, ne, g, k);
}

// trace at point (led, gp) of the six modes at slot[off .. off+5], mode 1
// first, as trace6 sums them
template <class Basis>
__device__ __forceinline__ real p2_slot_trace(const Basis& B, const real* slot, int off, int led, int gp) {
  const real* phi = B.phi_edge[led][gp];
  real t = slot[off];
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) t = t + slot[off + k] * phi[k];
  return t;
}

// Hybrid friction factor from the element-mean depth of a slot
template <bool kNonlin>
__device__ __forceinline__ real p2_hybrid(const Physics& P, const real* sl) {
#ifdef DGSWEM_MIXED
  const real depth_c = sl[3 * kP2Modes];  // depth mode 1
#else
  const real depth_c = sl[3 * kP2Modes] + sl[0];
#endif
  const real fh_c = real(1) / (kNonlin ? depth_c : real(P.nleq) * depth_c + real(P.leq));
  return pow(real(1) + pow(real(P.hbreak) * fh_c, real(P.ftheta)), real(P.fgamma / P.ftheta));
}

// Flux (F, G, H) at Lobatto point I of edge task tk into o[0..2]: the LLF
// flux in the in/ex orientation for an interior edge, else the land / ocean
// ghost state and its flux
template <bool kNonlin>
__device__ __forceinline__ void p2_tile_edge_point(const P2Args& A, const P2EdgeBasis& B, const real* qs,
                                                   const real* geo, uint2 tk, int I, real* o) {
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const unsigned fl = tk.x, kind = fl & 7u;
  const int sin = (fl >> TaskBits::kInSlot) & 511, sex = (fl >> TaskBits::kExSlot) & 511;
  const int led_in = (fl >> TaskBits::kLedIn) & 3, led_ex = (fl >> TaskBits::kLedEx) & 3;
  const bool flip = (fl >> TaskBits::kFlip) & 1u;
  const int owner = flip ? sex : sin, oled = flip ? led_ex : led_in;
  real nx = geo[(EGeo::kNx + oled) * kP2Tile + owner], ny = geo[(EGeo::kNy + oled) * kP2Tile + owner];
  if (flip) { nx = -nx; ny = -ny; }
  const real* si = qs + sin * kP2SlotStride;
  const real zi = p2_slot_trace(B, si, 0, led_in, I), xi = p2_slot_trace(B, si, kP2Modes, led_in, I);
  const real yi = p2_slot_trace(B, si, 2 * kP2Modes, led_in, I);
  const real wi = p2_slot_trace(B, si, 3 * kP2Modes, led_in, I);
  real hi, hti;
  trace_depth<kNonlin>(P, zi, wi, hi, hti);
  if (kind == kInterior) {
    const int J = kP2Egp - 1 - I;
    const real* sx = qs + sex * kP2SlotStride;
    const real zx = p2_slot_trace(B, sx, 0, led_ex, J), xx = p2_slot_trace(B, sx, kP2Modes, led_ex, J);
    const real yx = p2_slot_trace(B, sx, 2 * kP2Modes, led_ex, J);
    const real wx = p2_slot_trace(B, sx, 3 * kP2Modes, led_ex, J);
    real hx, htx;
    trace_depth<kNonlin>(P, zx, wx, hx, htx);
    const Flux3T<real> f =
        llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hx, hti, htx, real(1), real(1), nx, ny, real(P.g));
    o[0] = f.f; o[1] = f.g; o[2] = f.h;
    return;
  }
  // ghost state: land reflects the normal momentum (land_edge_hydro.F:201-218);
  // ocean takes the harmonic elevation with the depth-positivity fix
  // (ocean_edge_hydro.F:148-177, 255-259; FP64 in every variant)
  real zx = zi, xx = xi, yx = yi, htx = hti;
  if (kind == kOcean) {
    const int list = (int)tk.y;
    double zsum = 0.0;
    for (int f = 0; f < m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * cB2.xegp[I]);
    }
    const double hid = hi;
    if (zsum * P.ifnlfa + hid <= 0) zsum = fabs(hid) + P.h0;
    zx = (real)zsum;
    htx = depth<kNonlin>(P, zx, hi);
  } else {
    const real tx = -ny, ty = nx;
    const real qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const real qne = -qn, qte = qt, den = real(1) / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  }
  const Flux3T<real> f =
      llf<kNonlin, real>(P, zi, zx, xi, xx, yi, yx, hi, hi, hti, htx, real(1), real(1), nx, ny, real(P.g));
  o[0] = f.f; o[1] = f.g; o[2] = f.h;
}

template <bool kNonlin>
__global__ void __launch_bounds__(kP2TileThreads, 2) p2_tile(const __grid_constant__ P2Args A) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const int ne = m.ne;
  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  const int tile0 = m.tile_elem_ptr[tile];
  const int n = m.tile_elem_ptr[tile + 1] - tile0;
  const int hbeg = m.tile_halo_ptr[tile], nh = m.tile_halo_ptr[tile + 1] - hbeg;
  const int tbeg = m.tile_task_ptr[tile], ntask = m.tile_task_ptr[tile + 1] - tbeg;
  const P2Layout L = p2_layout(m.max_halo, m.max_tasks);
  P2EdgeBasis& B = *reinterpret_cast<P2EdgeBasis*>(smem_raw);
  real* qs = reinterpret_cast<real*>(smem_raw + L.qs);
  real* geo = reinterpret_cast<real*>(smem_raw + L.geo);
  real* frc = reinterpret_cast<real*>(smem_raw + L.frc);  // cori, fric, wx[3], wy[3], pr[3]: [kRows][kP2Tile]
  real* vol = reinterpret_cast<real*>(smem_raw + L.vol);
  real* res = reinterpret_cast<real*>(smem_raw + L.res);
  unsigned* sinfo = reinterpret_cast<unsigned*>(smem_raw + L.info);  // [einfo | eslot][kP2Tile]
  uint2* stasks = reinterpret_cast<uint2*>(smem_raw + L.tasks);
  const real* G = egeo_r(m);
  const bool hybrid = P.iflinbf == 0 && P.ifhybf == 1;
  for (int i = tid; i < 3 * kP2Egp * kP2Modes; i += kP2TileThreads) {
    const int row = i / kP2Modes, k = i - row * kP2Modes;
    (&B.phi_edge[0][0][0])[row * kP2EbRow + k] = (&cB2R.phi_edge[0][0][0])[i];
  }
  // ---- phase 1: slots, geometry rows, edge info, task words, forcing ----
  // Exact copies go by cp.async (issued back to back, one wait); the halo
  // ids are fetched first, the forcing gathers (node ids, then the nodal
  // fields) last, so their round trips overlap the copies in flight.
  const int hj = tid - kP2Tile;
  const int hg = (hj >= 0 && hj < nh) ? m.tile_halo[hbeg + hj] : -1;
  {
    constexpr unsigned rb = sizeof(real);
    const unsigned geo_s = smem_addr(geo);
    for (int j = tid; j < EGeo::kSmemRows * kP2Tile; j += kP2TileThreads) {
      const int r = j / kP2Tile, w = j - r * kP2Tile;
      if (w < n && (r != EGeo::kNbar || m.manning)) {
        if (rb == 8)
          cp_async8_s(geo_s + (unsigned)(r * kP2Tile + w) * rb, G + (size_t)r * ne + tile0 + w);
        else
          cp_async4_s(geo_s + (unsigned)(r * kP2Tile + w) * rb, G + (size_t)r * ne + tile0 + w);
      }
    }
  }
  if (tid < n) {
    cp_async4(sinfo + tid, m.einfo + tile0 + tid);
    cp_async4(sinfo + kP2Tile + tid, m.eslot + tile0 + tid);
  }
  for (int j = tid; j < ntask; j += kP2TileThreads) cp_async8(stasks + j, m.tile_tasks + tbeg + j);
  for (int j = tid; j < kP2Tile + nh; j += kP2TileThreads) {
    if (j < kP2Tile && j >= n) continue;
    const int g = j < kP2Tile ? tile0 + j : (j == tid ? hg : m.tile_halo[hbeg + j - kP2Tile]);
    real* sl = qs + j * kP2SlotStride;
#ifdef DGSWEM_MIXED
    p2_slot_store(A, g, sl);  // FP32 values and the depth modes: through registers
#else
    const unsigned d = smem_addr(sl);
#pragma unroll
    for (int c = 0; c < 3 * kP2Modes; ++c) cp_async8_s(d + 8u * c, A.qin + (size_t)c * ne + g);
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) cp_async8_s(d + 8u * (3 * kP2Modes + k), m.hb + (size_t)k * ne + g);
#endif
  }
  {  // the last kP2Tile threads: the forcing terms of the tile's elements
    const int j = tid - (kP2TileThreads - kP2Tile);
    if (j >= 0 && j < n) {
      const P2Frc F = p2_force(A, tile0 + j);
      frc[0 * kP2Tile + j] = F.cori;
      frc[1 * kP2Tile + j] = F.fric;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        frc[(2 + a) * kP2Tile + j] = F.wx[a];
        frc[(5 + a) * kP2Tile + j] = F.wy[a];
        frc[(8 + a) * kP2Tile + j] = F.pr[a];
      }
    }
  }
  cp_async_wait_all();
  // hybrid friction factor of tile element tid from the slot it copied
  if (hybrid && tid < n) geo[SGeo::kHyb * kP2Tile + tid] = p2_hybrid<kNonlin>(P, qs + tid * kP2SlotStride);
  __syncthreads();

  // ---- phase 2: edge points (edge task, Lobatto point), then area points ----
  // (the edge items padded to whole warps: a warp's area points share the
  // point i, so its basis values are uniform constant-memory loads)
  const int nep = kP2Egp * ntask, nep_pad = (nep + 31) & ~31;
  for (int w = tid; w < nep_pad + kP2Agp * kP2Tile; w += kP2TileThreads) {
    if (w < nep_pad) {
      if (w < nep) {
        const int ti = w / kP2Egp, I = w - kP2Egp * ti;
        p2_tile_edge_point<kNonlin>(A, B, qs, geo, stasks[ti], I, res + (size_t)ti * kP2ResStride + I * 3);
      }
      continue;
    }
    const int wa = w - nep_pad, i = wa / kP2Tile, el = wa - i * kP2Tile;
    if (el >= n) continue;
    const real* sl = qs + el * kP2SlotStride;
    real q[3 * kP2Modes], wm[kP2Modes];
#pragma unroll
    for (int c = 0; c < 3 * kP2Modes; ++c) q[c] = sl[c];
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) wm[k] = sl[3 * kP2Modes + k];
    const real drdx = geo[EGeo::kDrdx * kP2Tile + el], dsdx = geo[EGeo::kDsdx * kP2Tile + el];
    const real drdy = geo[EGeo::kDrdy * kP2Tile + el], dsdy = geo[EGeo::kDsdy * kP2Tile + el];
    const real hyb = hybrid ? geo[SGeo::kHyb * kP2Tile + el] : real(1);
    P2Frc F;
    F.cori = frc[0 * kP2Tile + el];
    F.fric = frc[1 * kP2Tile + el];
    F.nbar = m.manning ? geo[EGeo::kNbar * kP2Tile + el] : real(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const bool met = P.nws != 0;
      F.wx[a] = met ? frc[(2 + a) * kP2Tile + el] : real(0);
      F.wy[a] = met ? frc[(5 + a) * kP2Tile + el] : real(0);
      F.pr[a] = met ? frc[(8 + a) * kP2Tile + el] : real(0);
    }
    real v[kP2Vol];
    p2_volume<kNonlin>(A, q, wm, drdx, dsdx, drdy, dsdy, hyb, F, i, v);
#pragma unroll
    for (int r = 0; r < kP2Vol; ++r) vol[(r * kP2Agp + i) * kP2Tile + el] = v[r];
  }
  __syncthreads();

  // ---- phase 3: per (element, mode) sums in p2_elements' order, SSP ----
  for (int w = tid; w < kP2Modes * kP2Tile; w += kP2TileThreads) {
    const int K = w / kP2Tile, el = w - K * kP2Tile;
    if (el >= n) continue;
    const int e = tile0 + el;
    // the SSP combination's state operands, loaded before the sums
    const bool hist0 = A.irk > 1;
    double qc[3], qh0[3], rh0[3];
#pragma unroll
    for (int V = 0; V < 3; ++V) {
      const size_t c = (size_t)(kP2Modes * V + K) * ne + e;
#ifdef DGSWEM_MIXED
      qc[V] = A.qin[c];
#else
      qc[V] = qs[el * kP2SlotStride + kP2Modes * V + K];  // the slot holds qin exactly
#endif
      qh0[V] = (hist0 && A.a[0] != 0.0) ? A.qhist[0][c] : 0.0;
      rh0[V] = (hist0 && A.b[0] != 0.0) ? A.rhist[0][c] : 0.0;
    }
    const unsigned info = sinfo[el], slots = sinfo[kP2Tile + el];
    // The sums and their weights in FP64 in every variant: the mixed form
    // rounds only the operands (fluxes, volume terms) to FP32.  With FP32
    // weights the hydrostatic pressure's edge and volume integrals no longer
    // cancel to FP32 precision, and on a fine mesh the residual drives a
    // spurious flow (config 3 at 8M elements after 5000 steps: 1.5e-5 m,
    // against 3.5e-6 m with FP64 weights and sums).
#ifdef DGSWEM_MIXED
    using acc_t = double;
    const BasisP2& CW = cB2;
#else
    using acc_t = real;
    const BasisP2T<real>& CW = cB2R;
#endif
    acc_t rhs[3] = {0, 0, 0}, isum[3] = {0, 0, 0};
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int l = ei_order(info, s);
      const unsigned kind = ei_kind(info, l);
      if (kind == kNone) continue;
      const int ti = (slots >> (10 * l)) & kNoTask;
      const real* r = res + (size_t)ti * kP2ResStride;
      if (kind == kInterior) {
        const bool is_in = ei_flag(info, l) != 0;
        const acc_t edfac = geo[(EGeo::kEdfac + l) * kP2Tile + el];
        acc_t acc[3] = {0, 0, 0};
#pragma unroll
        for (int I = 0; I < kP2Egp; ++I) {
          const int j = is_in ? I : kP2Egp - 1 - I;
          const acc_t wk = edfac * (acc_t)CW.edgeq[l][j][K];
          // the in side subtracts: acc + (-wk) * v equals acc - wk * v exactly
          const acc_t ws = is_in ? -wk : wk;
          const acc_t v0 = r[I * 3], v1 = r[I * 3 + 1], v2 = r[I * 3 + 2];
          acc[0] = acc[0] + ws * v0;
          acc[1] = acc[1] + ws * v1;
          acc[2] = acc[2] + ws * v2;
        }
#pragma unroll
        for (int V = 0; V < 3; ++V) isum[V] = isum[V] + acc[V];
      } else {
        const acc_t areas = G[(size_t)EGeo::kAreas * ne + e];
        const acc_t xlen = G[(size_t)(EGeo::kXlen + l) * ne + e];
#pragma unroll
        for (int I = 0; I < kP2Egp; ++I) {
          const acc_t wk = acc_t(2) * CW.m_inv[K] / areas * xlen * CW.phi_edge[l][I][K] * CW.wegp[I];
          rhs[0] = rhs[0] - wk * (acc_t)r[I * 3];
          rhs[1] = rhs[1] - wk * (acc_t)r[I * 3 + 1];
          rhs[2] = rhs[2] - wk * (acc_t)r[I * 3 + 2];
        }
      }
    }
#pragma unroll
    for (int V = 0; V < 3; ++V) rhs[V] = rhs[V] + isum[V];  // add_internal_flux
    // the mode K and point i are the same across a warp: basis values from
    // constant memory (uniform loads), the shared-memory pipe kept for the
    // per-element operands
    const auto& C = CW;
    if (P.rainfall == 1) {
      const acc_t src = acc_t(7.0556e-6);
      for (int i = 0; i < kP2Agp; ++i) rhs[0] = rhs[0] + C.srfac[K][i] * src;
    }
    const acc_t drdx = geo[EGeo::kDrdx * kP2Tile + el], dsdx = geo[EGeo::kDsdx * kP2Tile + el];
    const acc_t drdy = geo[EGeo::kDrdy * kP2Tile + el], dsdy = geo[EGeo::kDsdy * kP2Tile + el];
#pragma unroll
    for (int i = 0; i < kP2Agp; ++i) {
      const real* vv = vol + i * kP2Tile + el;  // row r at vv[r * kP2Agp * kP2Tile]
      const acc_t sx = vv[6 * kP2Agp * kP2Tile], sy = vv[7 * kP2Agp * kP2Tile];
      if (K == 0) {
        rhs[1] = rhs[1] + C.srfac[0][i] * sx;
        rhs[2] = rhs[2] + C.srfac[0][i] * sy;
      } else {
        const acc_t dpx = C.drphi[K][i] * drdx + C.dsphi[K][i] * dsdx;
        const acc_t dpy = C.drphi[K][i] * drdy + C.dsphi[K][i] * dsdy;
        const acc_t xf = C.mw[K][i] * dpx;
        const acc_t yf = C.mw[K][i] * dpy;
        const acc_t sr = C.srfac[K][i];
        rhs[0] = rhs[0] + xf * (acc_t)vv[0] + yf * (acc_t)vv[kP2Agp * kP2Tile];
        rhs[1] = rhs[1] + xf * (acc_t)vv[2 * kP2Agp * kP2Tile] + yf * (acc_t)vv[3 * kP2Agp * kP2Tile] + sr * sx;
        rhs[2] = rhs[2] + xf * (acc_t)vv[4 * kP2Agp * kP2Tile] + yf * (acc_t)vv[5 * kP2Agp * kP2Tile] + sr * sy;
      }
    }
    // SSP-RK combination (DG_hydro_timestep.F:238-290) in FP64
    bool bad = false;
#pragma unroll
    for (int V = 0; V < 3; ++V) {
      const size_t c = (size_t)(kP2Modes * V + K) * ne + e;
      const double rk = (double)rhs[V];
      if (A.rout) A.rout[c] = rk;
      double acc = 0.0;
      if (hist0) {
        if (A.a[0] != 0.0) acc = acc + A.a[0] * qh0[V];
        if (A.b[0] != 0.0) acc = acc + A.b[0] * rh0[V];
      }
      for (int I = 1; I < A.irk; ++I) {
        const bool cur = I == A.irk - 1;
        if (A.a[I] != 0.0) acc = acc + A.a[I] * (cur ? qc[V] : A.qhist[I][c]);
        if (A.b[I] != 0.0) acc = acc + A.b[I] * (cur ? rk : A.rhist[I][c]);
      }
      if (!hist0) {
        if (A.a[0] != 0.0) acc = acc + A.a[0] * qc[V];
        if (A.b[0] != 0.0) acc = acc + A.b[0] * rk;
      }
      bad = bad || isnan(acc);
      A.qout[c] = acc;
    }
    if (bad) atomicOr(A.err, 1u);
  }
}

// write_results.F:14-170 at p=2 (six modes at the element corners) + NODECODE
__global__ void p2_modal2nodal(MeshView m, const double* __restrict__ q, double nleq, double leq, double* eta2,
                               double* uu2, double* vv2, int* nodecode) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.np) return;
  const int ne = m.ne;
  const BasisP2& B = cB2;
  double area_sum = 0.0;
  for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
    const int e = m.star[p];
    const int a = m.nm[e], b = m.nm[(size_t)ne + e], c = m.nm[(size_t)2 * ne + e];
    const double areas = (m.x[a] - m.x[c]) * (m.y[b] - m.y[c]) + (m.x[c] - m.x[b]) * (m.y[a] - m.y[c]);
    area_sum = area_sum + 0.5 * areas;
  }
  double et = 0.0, uu = 0.0, vv = 0.0;
  for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
    const int e = m.star[p];
    const int a = m.nm[e], b = m.nm[(size_t)ne + e], c = m.nm[(size_t)2 * ne + e];
    const int K = (a == n) ? 0 : (b == n) ? 1 : 2;
    double zd = q[e], xd = q[(size_t)6 * ne + e], yd = q[(size_t)12 * ne + e], hd = m.hb[e];
#pragma unroll
    for (int kk = 1; kk < kP2Modes; ++kk) {
      const double pc = B.phi_corner[K][kk];
      zd = zd + pc * q[(size_t)kk * ne + e];
      xd = xd + pc * q[(size_t)(6 + kk) * ne + e];
      yd = yd + pc * q[(size_t)(12 + kk) * ne + e];
      hd = hd + pc * m.hb[(size_t)kk * ne + e];
    }
    const double areas = (m.x[a] - m.x[c]) * (m.y[b] - m.y[c]) + (m.x[c] - m.x[b]) * (m.y[a] - m.y[c]);
    const double w = 0.50 * areas / area_sum;
    const double fh = 1.0 / (nleq * (zd + hd) + leq);
    et = et + w * zd;
    uu = uu + w * xd * fh;
    vv = vv + w * yd * fh;
  }
  const int out = m.node_perm[n];
  if (eta2) eta2[out] = et;
  if (uu2) uu2[out] = uu;
  if (vv2) vv2[out] = vv;
  if (nodecode) nodecode[out] = 1;
}

// ZE/QX/QY(DOFH=6, NE) of the input order <-> state rows of the device order
__global__ void p2_fortran_to_soa(const double* __restrict__ f, double* __restrict__ q, int ne, int var,
                                  const int* __restrict__ perm) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const int e = perm[i];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) q[(size_t)(kP2Modes * var + k) * ne + i] = f[(size_t)kP2Modes * e + k];
}

__global__ void p2_soa_to_fortran(const double* __restrict__ q, double* __restrict__ f, int ne, int var,
                                  const int* __restrict__ inv) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  const int i = inv[e];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) f[(size_t)kP2Modes * e + k] = q[(size_t)(kP2Modes * var + k) * ne + i];
}

size_t p2_tile_smem(int max_halo, int max_tasks) { return p2_layout(max_halo, max_tasks).bytes; }

void set_basis_p2(const BasisP2& b) {
  cudaMemcpyToSymbol(cB2, &b, sizeof(b));
  BasisP2T<real> r;
  const double* src = reinterpret_cast<const double*>(&b);
  real* dst = reinterpret_cast<real*>(&r);
  for (size_t i = 0; i < sizeof(b) / sizeof(double); ++i) dst[i] = (real)src[i];
  cudaMemcpyToSymbol(cB2R, &r, sizeof(r));
}

void launch_p2_stage(const P2Args& a, bool nonlin, cudaStream_t s) {
  if (a.ntile > 0) {  // the tile kernel
    const size_t smem = p2_layout(a.m.max_halo, a.m.max_tasks).bytes;
    auto* k = nonlin ? p2_tile<true> : p2_tile<false>;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k<<<(unsigned)a.ntile, kP2TileThreads, smem, s>>>(a);
    return;
  }
  const unsigned ge = (unsigned)(((long long)kP2Egp * a.nedge + 127) / 128);
  const unsigned gl = (unsigned)((a.ne_act + 127) / 128);
  if (nonlin) {
    if (ge) p2_edges<true><<<ge, 128, 0, s>>>(a);
    if (gl) p2_elements<true><<<gl, 128, 0, s>>>(a);
  } else {
    if (ge) p2_edges<false><<<ge, 128, 0, s>>>(a);
    if (gl) p2_elements<false><<<gl, 128, 0, s>>>(a);
  }
}

void launch_p2_modal2nodal(const MeshView& m, const double* q, double nleq, double leq, double* eta2, double* uu2,
                           double* vv2, int* nodecode, cudaStream_t s) {
  p2_modal2nodal<<<(unsigned)((m.np + 127) / 128), 128, 0, s>>>(m, q, nleq, leq, eta2, uu2, vv2, nodecode);
}

void launch_p2_layout(bool to_device, const double* src, double* dst, int ne, int var, const int* map,
                      cudaStream_t s) {
  const unsigned g = (unsigned)((ne + 127) / 128);
  if (to_device)
    p2_fortran_to_soa<<<g, 128, 0, s>>>(src, dst, ne, var, map);
  else
    p2_soa_to_fortran<<<g, 128, 0, s>>>(src, dst, ne, var, map);
}

}  // namespace DGSWEM_VARIANT
}  // namespace dgswem
