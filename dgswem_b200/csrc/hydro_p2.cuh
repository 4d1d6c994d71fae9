// hydro_p2.cuh -- the p=2 stage (six modes per variable, four Gauss-Lobatto
// points per edge, the six-point area rule), FP64: an edge kernel and an
// element kernel per RK stage.  Included after hydro_kernels.cuh (its LLF
// flux and depth) by kernels_p2_fast.cu / kernels_p2_strict.cu with
// DGSWEM_VARIANT set.  The arithmetic follows the p=1 kernels term for term,
// generalised over the modes and points as the reference's p-generic
// boundary-edge code (land_edge_hydro.F:144,273) is; the interior-edge sums
// run over every mode (the reference's internal_edge_hydro.F:306-318 sums
// modes 1-3 only, its p=2 defect).  No wetting/drying and no slope limiter
// at p=2 (both are p=1 only in the reference); land, ocean and interior
// edges; ICS=1.
#pragma once

namespace dgswem {
namespace DGSWEM_VARIANT {

__constant__ BasisP2 cB2;

// Traces of ZE, QX, QY and HB at one point from the six modes (state rows
// 6*var + k, bathymetry rows k), summed from mode 1 upwards as the
// reference's trace loops are (mode 1 is 1 at every point).
__device__ __forceinline__ void trace6(const double* __restrict__ q, const double* __restrict__ hb, int ne,
                                       int e, const double* phi, double& z, double& u, double& v, double& h) {
  z = q[e];
  u = q[(size_t)6 * ne + e];
  v = q[(size_t)12 * ne + e];
  h = hb[e];
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) {
    z = z + q[(size_t)k * ne + e] * phi[k];
    u = u + q[(size_t)(6 + k) * ne + e] * phi[k];
    v = v + q[(size_t)(12 + k) * ne + e] * phi[k];
    h = h + hb[(size_t)k * ne + e] * phi[k];
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
  const BasisP2& B = cB2;
  const int ne = m.ne;
  const int e = A.edges[2 * ed], l = A.edges[2 * ed + 1];
  const unsigned info = m.einfo[e], kind = ei_kind(info, l);
  const double nx = m.egeo[(size_t)(EGeo::kNx + l) * ne + e], ny = m.egeo[(size_t)(EGeo::kNy + l) * ne + e];
  double zi, xi, yi, hi;
  trace6(A.qin, m.hb, ne, e, B.phi_edge[l][I], zi, xi, yi, hi);
  const double hti = depth<kNonlin>(P, zi, hi);
  double* o = A.ef + ((size_t)(e * 3 + l) * kP2Egp + I) * 3;
  if (kind == kInterior) {
    const int ex = m.link[(size_t)l * ne + e], lx = (int)ei_nled(info, l), J = kP2Egp - 1 - I;
    double zx, xx, yx, hx;
    trace6(A.qin, m.hb, ne, ex, B.phi_edge[lx][J], zx, xx, yx, hx);
    const double htx = depth<kNonlin>(P, zx, hx);
    const Flux3 f = llf<kNonlin, double>(P, zi, zx, xi, xx, yi, yx, hi, hx, hti, htx, 1.0, 1.0, nx, ny, P.g);
    o[0] = f.f; o[1] = f.g; o[2] = f.h;
    double* ox = A.ef + ((size_t)(ex * 3 + lx) * kP2Egp + J) * 3;
    ox[0] = f.f; ox[1] = f.g; ox[2] = f.h;
    return;
  }
  // ghost state: land reflects the normal momentum (land_edge_hydro.F:201-218);
  // ocean takes the harmonic elevation with the depth-positivity fix
  // (ocean_edge_hydro.F:148-177, 255-259) and the interior momentum
  double zx = zi, xx = xi, yx = yi, htx = hti;
  if (kind == kOcean) {
    const int list = m.link[(size_t)l * ne + e];
    double zsum = 0.0;
    for (int f = 0; f < m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * B.xegp[I]);
    }
    if (zsum * P.ifnlfa + hi <= 0) zsum = fabs(hi) + P.h0;
    zx = zsum;
    htx = depth<kNonlin>(P, zx, hi);
  } else {
    const double tx = -ny, ty = nx;
    const double qn = xi * nx + yi * ny, qt = xi * tx + yi * ty;
    const double qne = -qn, qte = qt, den = 1.0 / (nx * ty - ny * tx);
    xx = (ty * qne - ny * qte) * den;
    yx = (-tx * qne + nx * qte) * den;
  }
  const Flux3 f = llf<kNonlin, double>(P, zi, zx, xi, xx, yi, yx, hi, hi, hti, htx, 1.0, 1.0, nx, ny, P.g);
  o[0] = f.f; o[1] = f.g; o[2] = f.h;
}


// Volume fluxes and sources at area point i of element e (rhs_dg_hydro.F:58-470
// with six modes): out = fx fy gx gy hx hy sx sy.  q: the element's 18 state
// values (row 6*var + k), hbe: its six bathymetry modes.
template <bool kNonlin>
__device__ __forceinline__ void p2_volume(const P2Args& A, const double* q, const double* hbe, double drdx,
                                          double dsdx, double drdy, double dsdy, double hyb, int e, int i,
                                          double out[8]) {
  const MeshView& m = A.m;
  const Physics& P = A.ph;
  const BasisP2& C = cB2;
  const int ne = m.ne;
  const double NLEQ = kNonlin ? 1.0 : P.nleq, LEQ = kNonlin ? 0.0 : P.leq;
  const double cori = m.cori ? m.cori[e] : P.cori;
  double fric = m.fric ? m.fric[e] : P.fric;
  double zq = q[0], uq = q[6], vq = q[12];
  double hq = hbe[0] * C.phi_area[0][i];
#pragma unroll
  for (int k = 1; k < kP2Modes; ++k) hq = hq + hbe[k] * C.phi_area[k][i];
  double dhx = 0, dhy = 0;
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
  const double depth = zq + hq;
  const double f1 = kNonlin ? 1.0 : NLEQ + LEQ * hq;
  const double fx = uq * f1 * 1.0, fy = vq * f1;
  const double fu = kNonlin ? uq : NLEQ * uq, fv = kNonlin ? vq : NLEQ * vq;
  const double fg = P.nleqg * zq * 1;
  const double fh = 1.0 / (kNonlin ? depth : NLEQ * depth + LEQ);
  const double u = uq * fh, v = vq * fh;
  const double huu = fu * u, hvv = fv * v, huv = fu * v;
  const double gh2 = kNonlin ? fg * (0.5 * zq + hq) : fg * (0.5 * zq + hq) + P.fg_l * zq;
  const double gx = (huu + gh2) * 1.0, gy = huv;
  const double hx = huv * 1.0, hy = hvv + gh2;
  if (m.manning) {
    const double nbar = m.egeo[(size_t)EGeo::kNbar * ne + e];
    fric = P.g * (nbar * nbar) / cube_root(depth);
    if (fric < P.cf) fric = P.cf;
  }
  double tau = fric;
  if (P.iflinbf == 0) {
    const double umag = sqrt(u * u + v * v);
    tau = tau * umag * fh;
    if (P.ifhybf == 1) tau = tau * hyb;
    tau = fmin(tau, P.tau_cap);
  }
  double sx = -(tau * uq) + fg * dhx * 1.0 + cori * vq;
  double sy = -(tau * vq) + fg * dhy - cori * uq;
  if (P.nws != 0) {
    // met_forcing.F:49-66: the nodal fields scaled by the stage's ramp
    const double drpsi[3] = {-0.5, 0.5, 0.0}, dspsi[3] = {-0.5, 0.0, 0.5};
    double dpsidx[3], dpsidy[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dpsidx[a] = drpsi[a] * drdx + dspsi[a] * dsdx;
      dpsidy[a] = drpsi[a] * drdy + dspsi[a] * dsdy;
    }
    const double fw = 1.0 / f1, r = A.ramp ? *A.ramp : A.rampdg;
    const int n0 = m.nm[e], n1 = m.nm[(size_t)ne + e], n2 = m.nm[(size_t)2 * ne + e];
    const double wx0 = r * A.wsx[n0], wx1 = r * A.wsx[n1], wx2 = r * A.wsx[n2];
    const double wy0 = r * A.wsy[n0], wy1 = r * A.wsy[n1], wy2 = r * A.wsy[n2];
    const double p0 = r * A.pr[n0], p1 = r * A.pr[n1], p2 = r * A.pr[n2];
    sx = sx + fw * (wx0 * C.psi[0][i] + wx1 * C.psi[1][i] + wx2 * C.psi[2][i]) -
         P.g * 1.0 * depth * (p0 * dpsidx[0] + p1 * dpsidx[1] + p2 * dpsidx[2]);
    sy = sy + fw * (wy0 * C.psi[0][i] + wy1 * C.psi[1][i] + wy2 * C.psi[2][i]) -
         P.g * depth * (p0 * dpsidy[0] + p1 * dpsidy[1] + p2 * dpsidy[2]);
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
  const BasisP2& B = cB2;
  const int ne = m.ne;
  double q[3 * kP2Modes], hbe[kP2Modes];
#pragma unroll
  for (int c = 0; c < 3 * kP2Modes; ++c) q[c] = A.qin[(size_t)c * ne + e];
#pragma unroll
  for (int k = 0; k < kP2Modes; ++k) hbe[k] = m.hb[(size_t)k * ne + e];
  const double drdx = m.egeo[(size_t)EGeo::kDrdx * ne + e], dsdx = m.egeo[(size_t)EGeo::kDsdx * ne + e];
  const double drdy = m.egeo[(size_t)EGeo::kDrdy * ne + e], dsdy = m.egeo[(size_t)EGeo::kDsdy * ne + e];
  double hyb = 1.0;
  if (P.iflinbf == 0 && P.ifhybf == 1) {
    const double depth_c = hbe[0] + q[0];
    const double fh_c = 1.0 / (kNonlin ? depth_c : P.nleq * depth_c + P.leq);
    hyb = pow(1.0 + pow(P.hbreak * fh_c, P.ftheta), P.fgamma / P.ftheta);
  }
  // all three variables' sums at once (no per-point volume array): each
  // (variable, mode) sum takes the same terms in the same order as above
  const unsigned info = m.einfo[e];
  double rhs[3][kP2Modes], isum[3][kP2Modes];
#pragma unroll
  for (int V = 0; V < 3; ++V)
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) { rhs[V][k] = 0.0; isum[V][k] = 0.0; }
  for (int s = 0; s < 3; ++s) {
    const int l = ei_order(info, s);
    const unsigned kind = ei_kind(info, l);
    if (kind == kNone) continue;
    const double* ef = A.ef + (size_t)(e * 3 + l) * kP2Egp * 3;
    if (kind == kInterior) {
      const bool is_in = ei_flag(info, l) != 0;
      const double edfac = m.egeo[(size_t)(EGeo::kEdfac + l) * ne + e];
      double acc[3][kP2Modes];
#pragma unroll
      for (int V = 0; V < 3; ++V)
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) acc[V][k] = 0.0;
      for (int I = 0; I < kP2Egp; ++I) {
        const int j = is_in ? I : kP2Egp - 1 - I;
        const double v0 = ef[j * 3], v1 = ef[j * 3 + 1], v2 = ef[j * 3 + 2];
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) {
          const double wk = edfac * B.edgeq[l][j][k];
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
      const double areas = m.egeo[(size_t)EGeo::kAreas * ne + e];
      const double xlen = m.egeo[(size_t)(EGeo::kXlen + l) * ne + e];
      for (int I = 0; I < kP2Egp; ++I) {
        const double v0 = ef[I * 3], v1 = ef[I * 3 + 1], v2 = ef[I * 3 + 2];
#pragma unroll
        for (int k = 0; k < kP2Modes; ++k) {
          const double wk = 2.0 * B.m_inv[k] / areas * xlen * B.phi_edge[l][I][k] * B.wegp[I];
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
    const double src = 7.0556e-6;
    for (int i = 0; i < kP2Agp; ++i)
#pragma unroll
      for (int k = 0; k < kP2Modes; ++k) rhs[0][k] = rhs[0][k] + B.srfac[k][i] * src;
  }
  for (int i = 0; i < kP2Agp; ++i) {
    double vol[8];
    p2_volume<kNonlin>(A, q, hbe, drdx, dsdx, drdy, dsdy, hyb, e, i, vol);
    rhs[1][0] = rhs[1][0] + B.srfac[0][i] * vol[6];
    rhs[2][0] = rhs[2][0] + B.srfac[0][i] * vol[7];
#pragma unroll
    for (int k = 1; k < kP2Modes; ++k) {
      const double dpx = B.drphi[k][i] * drdx + B.dsphi[k][i] * dsdx;
      const double dpy = B.drphi[k][i] * drdy + B.dsphi[k][i] * dsdy;
      const double xf = B.mw[k][i] * dpx;
      const double yf = B.mw[k][i] * dpy;
      const double sr = B.srfac[k][i];
      rhs[0][k] = rhs[0][k] + xf * vol[0] + yf * vol[1];
      rhs[1][k] = rhs[1][k] + xf * vol[2] + yf * vol[3] + sr * vol[6];
      rhs[2][k] = rhs[2][k] + xf * vol[4] + yf * vol[5] + sr * vol[7];
    }
  }
  // SSP-RK combination (DG_hydro_timestep.F:238-290); zero coefficients skipped
  bool bad = false;
  const bool hist0 = A.irk > 1;
#pragma unroll
  for (int V = 0; V < 3; ++V)
#pragma unroll
    for (int k = 0; k < kP2Modes; ++k) {
      const int c = kP2Modes * V + k;
      const double rk = rhs[V][k];
      if (A.rout) A.rout[(size_t)c * ne + e] = rk;
      const double qc = q[c];
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

void set_basis_p2(const BasisP2& b) { cudaMemcpyToSymbol(cB2, &b, sizeof(b)); }

void launch_p2_stage(const P2Args& a, bool nonlin, cudaStream_t s) {
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
