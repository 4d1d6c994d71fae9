// adjoint.cu -- hand-written discrete adjoint of one RK stage of the p=1 DG
// hydro step (no counterpart in the reference).
//
// The forward stage is L(q; n, HB): edge fluxes (LLF, numerical_flux.F:750-914)
// at the Lobatto points of every edge, volume fluxes and sources
// (rhs_dg_hydro.F:58-470) at the area points, summed with the basis weights
// of the stage kernel.  This file differentiates that map in reverse mode:
// lam += (dL/dq)^T nu and the parameter gradients for the element-mean
// Manning n and the bathymetry modes HB.  Non-smooth points take the branch
// the forward took at the same state (the LLF wave-speed maximum, the
// Manning floor CF, the friction cap 0.9/DT, the ocean depth-positivity fix).
//
// Scope: NLEQ=1 (finite amplitude), ICS=1, land and ocean edges (any other
// kind is rejected before launch), slope limiter 5 and WETDRY with their
// branches frozen at the forward's (node_arg .. elem_bound_scatter below;
// the stage's dry elements lose their volume terms and the dry-side edge
// rules replay the forward's choice), linear, quadratic or Manning friction
// (not hybrid), NWS 0/1.
//
// Deterministic without atomics: edge_vjp evaluates each edge point once
// and writes each side's trace cotangents to that element's own slots of a
// per-element buffer (one writer per slot); elem_vjp adds the volume terms
// and gathers the buffer, so each element's outputs are written by its own
// thread.
#include "hydro_device.cuh"

namespace dgswem {
namespace adj {

__constant__ BasisP1 cB;

void set_basis(const BasisP1& b) { cudaMemcpyToSymbol(cB, &b, sizeof(b)); }

// Trace of ZE, QX, QY (q: 9 modal values) and HB (3) at edge point (led, j).
__device__ __forceinline__ void trace(const double* q, const double* hb, int led, int j, double t[4]) {
  const double p1 = cB.phi_edge[led][j][1], p2 = cB.phi_edge[led][j][2];
  t[0] = q[0] + q[1] * p1 + q[2] * p2;
  t[1] = q[3] + q[4] * p1 + q[5] * p2;
  t[2] = q[6] + q[7] * p1 + q[8] * p2;
  t[3] = hb[0] + hb[1] * p1 + hb[2] * p2;
}

// Reverse mode of the LLF flux (NLEQ=1, ICS=1) at in-side trace a and
// ex-side trace b (ZE, QX, QY, HB each), normal (nx, ny), gravity G, given
// the cotangent c of (F, G, H).  da, db receive the cotangents of the traces.
__device__ void llf_vjp(const double a[4], const double b[4], double nx, double ny, double G, const double c[3],
                        double da[4], double db[4]) {
  const double* s[2] = {a, b};
  double* d[2] = {da, db};
  double H[2], iH[2], un[2], cc[2], aa[2];
  for (int k = 0; k < 2; ++k) {
    H[k] = s[k][0] + s[k][3];
    iH[k] = 1.0 / H[k];
    un[k] = (s[k][1] * nx + s[k][2] * ny) * iH[k];
    cc[k] = sqrt(G * H[k] * (ny * ny + nx * nx));
    aa[k] = fabs(un[k]);
  }
  const double eig = fmax(fmax(aa[0] + cc[0], aa[0]), fmax(aa[1] + cc[1], aa[1]));
  // cotangent of the wave-speed maximum; the jump terms
  const double deig = -0.5 * (c[0] * (b[0] - a[0]) + c[1] * (b[1] - a[1]) + c[2] * (b[2] - a[2]));
  for (int k = 0; k < 4; ++k) { da[k] = 0.0; db[k] = 0.0; }
  for (int v = 0; v < 3; ++v) {
    da[v] += 0.5 * eig * c[v];
    db[v] -= 0.5 * eig * c[v];
  }
  // which term the forward maximum took (first in evaluation order on ties)
  int side = -1;
  bool with_c = false;
  if (eig == aa[0] + cc[0]) { side = 0; with_c = true; }
  else if (eig == aa[0]) side = 0;
  else if (eig == aa[1] + cc[1]) { side = 1; with_c = true; }
  else side = 1;
  double dun[2] = {0.0, 0.0}, dH[2] = {0.0, 0.0};
  dun[side] += (un[side] >= 0.0 ? 1.0 : -1.0) * deig;
  if (with_c && cc[side] > 0.0) dH[side] += G * (ny * ny + nx * nx) / (2.0 * cc[side]) * deig;
  for (int k = 0; k < 2; ++k) {
    const double z = s[k][0], qx = s[k][1], qy = s[k][2], h = s[k][3], r = iH[k];
    // F = 0.5 (qx nx + qy ny) summed over both sides
    double dqx = 0.5 * nx * c[0], dqy = 0.5 * ny * c[0];
    // G: 0.5 ((qx u + gh2) nx + qx v ny); H: 0.5 (qx v nx + (qy v + gh2) ny)
    const double dA1 = 0.5 * nx * c[1];                  // qx*u = qx^2/H
    const double dA2 = 0.5 * ny * c[1] + 0.5 * nx * c[2];  // qx*v = qx qy/H
    const double dA3 = 0.5 * ny * c[2];                  // qy*v = qy^2/H
    const double dgh2 = 0.5 * nx * c[1] + 0.5 * ny * c[2];
    dqx += 2.0 * qx * r * dA1 + qy * r * dA2;
    dqy += qx * r * dA2 + 2.0 * qy * r * dA3;
    double dHk = dH[k] - (qx * qx * dA1 + qx * qy * dA2 + qy * qy * dA3) * (r * r);
    // un = (qx nx + qy ny) / H
    dqx += nx * r * dun[k];
    dqy += ny * r * dun[k];
    dHk -= un[k] * r * dun[k];
    // gh2 = G z (0.5 z + h)
    double dz = G * (z + h) * dgh2, dh = G * z * dgh2;
    // H = z + h
    dz += dHk;
    dh += dHk;
    d[k][0] += dz;
    d[k][1] += dqx;
    d[k][2] += dqy;
    d[k][3] += dh;
  }
}

// Mass flux F of the LLF at traces a (in) and b (ex): the value whose size
// and sign select internal_edge_hydro.F's dry-side rules.
__device__ double llf_mass(const double a[4], const double b[4], double nx, double ny, double G) {
  double eig = 0.0;
  const double* s[2] = {a, b};
  for (int k = 0; k < 2; ++k) {
    const double H = s[k][0] + s[k][3];
    const double un = (s[k][1] * nx + s[k][2] * ny) / H, c = sqrt(G * H * (ny * ny + nx * nx));
    eig = fmax(eig, fmax(fabs(un) + c, fabs(un)));
  }
  return 0.5 * ((a[1] + b[1]) * nx + (a[2] + b[2]) * ny) - 0.5 * eig * (b[0] - a[0]);
}

// Momentum (qx, qy) reflected across the edge (normal component negated,
// tangential kept: land_edge_hydro.F:201-218) and the transpose of that map
// applied to cotangents (dx, dy), added to (ax, ay).
__device__ __forceinline__ void reflect(double nx, double ny, double qx, double qy, double& rx, double& ry) {
  const double tx = -ny, ty = nx, qn = qx * nx + qy * ny, qt = qx * tx + qy * ty;
  rx = (ty * (-qn) - ny * qt) / (nx * ty - ny * tx);
  ry = (-tx * (-qn) + nx * qt) / (nx * ty - ny * tx);
}
__device__ __forceinline__ void reflect_t(double nx, double ny, double dx, double dy, double& ax, double& ay) {
  const double tx = -ny, ty = nx, den = 1.0 / (nx * ty - ny * tx);
  const double dqne = (ty * dx - tx * dy) * den, dqte = (-ny * dx + nx * dy) * den;
  ax += nx * (-dqne) + tx * dqte;
  ay += ny * (-dqne) + ty * dqte;
}

// Reverse mode of the volume fluxes and sources at area point i of element e
// (rhs_dg_hydro.F:58-470, NLEQ=1, ICS=1), given the cotangents dv of the
// eight terms (fx fy gx gy hx hy sx sy).  Adds the cotangents of the modal
// state (lam9), of HB (ghb) and of the element-mean Manning n (gn).
__device__ void volume_vjp(const AdjArgs& A, int e, int i, const double q[9], const double hb[3],
                           const double geo[6], double nbar, const double dv[8], double lam9[9], double ghb[3],
                           double& gn) {
  const Physics& P = A.ph;
  const MeshView& m = A.m;
  const double drdx = geo[0], dsdx = geo[1], drdy = geo[2], dsdy = geo[3];
  const double G = P.g;
  double phi[3], dx[3], dy[3];
  for (int k = 0; k < 3; ++k) {
    phi[k] = cB.phi_area[k][i];
    dx[k] = cB.drphi[k][i] * drdx + cB.dsphi[k][i] * dsdx;
    dy[k] = cB.drphi[k][i] * drdy + cB.dsphi[k][i] * dsdy;
  }
  double zq = 0, uq = 0, vq = 0, hq = 0, dhx = 0, dhy = 0;
  for (int k = 0; k < 3; ++k) {
    zq += q[k] * phi[k];
    uq += q[3 + k] * phi[k];
    vq += q[6 + k] * phi[k];
    hq += hb[k] * phi[k];
    dhx += hb[k] * dx[k];
    dhy += hb[k] * dy[k];
  }
  const double H = zq + hq, fh = 1.0 / H;
  const double cori = m.cori ? m.cori[e] : P.cori;
  // friction (forward branches re-evaluated at the same state)
  double fric = m.fric ? m.fric[e] : P.fric;
  bool floored = false;
  const double icbrt = m.manning ? 1.0 / cbrt(H) : 0.0;
  if (m.manning) {
    fric = G * (nbar * nbar) * icbrt;
    if (fric < P.cf) { fric = P.cf; floored = true; }
  }
  const double s = sqrt(uq * uq + vq * vq);
  double tau = fric;
  bool capped = false;
  if (P.iflinbf == 0) {
    tau = fric * s * fh * fh;
    if (tau > P.tau_cap) { tau = P.tau_cap; capped = true; }
  }
  // cotangents of the point values
  double dzq = 0, duq = 0, dvq = 0, dH = 0, ddhx = 0, ddhy = 0, dtau = 0;
  const double dfx = dv[0], dfy = dv[1], dgx = dv[2], dgy = dv[3], dhxf = dv[4], dhy_ = dv[5], dsx = dv[6],
               dsy = dv[7];
  duq += dfx;                                   // fx = uq
  dvq += dfy;                                   // fy = vq
  duq += 2.0 * uq * fh * dgx;                   // gx = uq^2/H + gh2
  dH -= uq * uq * fh * fh * dgx;
  const double dA = dgy + dhxf;                 // gy = hx = uq vq / H
  duq += vq * fh * dA;
  dvq += uq * fh * dA;
  dH -= uq * vq * fh * fh * dA;
  dvq += 2.0 * vq * fh * dhy_;                  // hy = vq^2/H + gh2
  dH -= vq * vq * fh * fh * dhy_;
  const double dgh2 = dgx + dhy_;               // gh2 = G zq (0.5 zq + hq)
  dzq += G * (zq + hq) * dgh2;
  double dhq = G * zq * dgh2;
  // sx = -tau uq + G zq dhx + cori vq ; sy = -tau vq + G zq dhy - cori uq
  dtau += -uq * dsx - vq * dsy;
  duq += -tau * dsx - cori * dsy;
  dvq += -tau * dsy + cori * dsx;
  dzq += G * dhx * dsx + G * dhy * dsy;
  ddhx += G * zq * dsx;
  ddhy += G * zq * dsy;
  if (P.nws != 0 && A.pr) {
    // pressure head terms -G H (sum p dpsi/dx), -G H (sum p dpsi/dy)
    const double drpsi[3] = {-0.5, 0.5, 0.0}, dspsi[3] = {-0.5, 0.0, 0.5};
    const int ne = m.ne;
    double px = 0.0, py = 0.0;
    for (int a = 0; a < 3; ++a) {
      const double p = A.rampdg * A.pr[m.nm[(size_t)a * ne + e]];
      px += p * (drpsi[a] * drdx + dspsi[a] * dsdx);
      py += p * (drpsi[a] * drdy + dspsi[a] * dsdy);
    }
    dH += -G * px * dsx - G * py * dsy;
  }
  // tau
  double dfric = 0.0;
  if (P.iflinbf == 0) {
    if (!capped) {
      dfric += s * fh * fh * dtau;
      if (s > 0.0) {
        const double is = 1.0 / s;
        duq += fric * uq * is * fh * fh * dtau;
        dvq += fric * vq * is * fh * fh * dtau;
      }
      dH += -2.0 * fric * s * fh * fh * fh * dtau;
    }
  } else {
    dfric += dtau;
  }
  if (m.manning && !floored) {  // fric = G nbar^2 H^(-1/3)
    gn += 2.0 * G * nbar * icbrt * dfric;
    dH += -fric * fh * (1.0 / 3.0) * dfric;
  }
  dzq += dH;  // H = zq + hq
  dhq += dH;
  for (int k = 0; k < 3; ++k) {
    lam9[k] += phi[k] * dzq;
    lam9[3 + k] += phi[k] * duq;
    lam9[6 + k] += phi[k] * dvq;
    ghb[k] += phi[k] * dhq + dx[k] * ddhx + dy[k] * ddhy;
  }
}

// Edge part: one thread per (edge, Lobatto point) of the edge list
// A.edges (each interior edge once, from its in side, and each land / ocean
// edge): the flux at that point is differentiated with respect to both
// sides' traces (ZE, QX, QY, HB), from the cotangents of both elements'
// right-hand sides (or of the element's alone, through the ghost state), and
// each side's four values go to its own slot eb[e*36 + (3l + gp)*4 + c] --
// one writer per slot.  Slots of edges in no list stay zero.
// The reverse-mode kernels are latency bound: they are compiled for more
// resident warps than their unbounded allocations (124-162 registers)
// allow, at the price of a few hundred bytes of spills to L1-cached local
// memory -- about 96 registers a thread, the fastest of the bounds timed
// on the 1M-element wet/dry beach (gradient 6 % faster than unbounded).
__global__ void __launch_bounds__(256, 3) edge_vjp(const __grid_constant__ AdjArgs A) {
  const MeshView& m = A.m;
  const int ne = m.ne;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3LL * A.nedge) return;
  const int ed = (int)(t / 3), I = (int)(t - 3LL * ed);
  const int e = A.edges[2 * ed], l = A.edges[2 * ed + 1];
  const Physics& P = A.ph;
  auto eg = [&](int row, int el) { return m.egeo[(size_t)row * ne + el]; };
  const unsigned info = m.einfo[e];
  const unsigned kind = ei_kind(info, l);
  const double nx = eg(EGeo::kNx + l, e), ny = eg(EGeo::kNy + l, e);
  if (kind == kInterior) {  // e is the in side
    const int ex = m.link[(size_t)l * ne + e], lx = (int)ei_nled(info, l);
    double* oi = A.eb + (size_t)e * 36 + (3 * l + I) * 4;
    double* ox = A.eb + (size_t)ex * 36 + (3 * lx + (2 - I)) * 4;
    const int wi = A.wd[e], wx = A.wd[ex];
    double da[4] = {0, 0, 0, 0}, db[4] = {0, 0, 0, 0};
    if (wi != 0 || wx != 0) {  // an edge between two dry elements adds nothing
      double qi[9], qx[9], hi[3], hx[3];
      for (int c = 0; c < 9; ++c) { qi[c] = A.q[(size_t)c * ne + e]; qx[c] = A.q[(size_t)c * ne + ex]; }
      for (int k = 0; k < 3; ++k) { hi[k] = m.hb[(size_t)k * ne + e]; hx[k] = m.hb[(size_t)k * ne + ex]; }
      double ta[4], tb[4];
      trace(qi, hi, l, I, ta);
      trace(qx, hx, lx, 2 - I, tb);
      const double efi = eg(EGeo::kEdfac + l, e), efx = eg(EGeo::kEdfac + lx, ex);
      // cotangents of F, G_in, H_in, G_ex, H_ex (the in side's sums subtract,
      // the ex side's add)
      double cF = 0, cGi = 0, cHi = 0, cGx = 0, cHx = 0;
      for (int k = 0; k < 3; ++k) {
        const double wi_k = efi * cB.edgeq[l][I][k], wx_k = efx * cB.edgeq[lx][2 - I][k];
        cF += -wi_k * A.nu[(size_t)k * ne + e] + wx_k * A.nu[(size_t)k * ne + ex];
        cGi -= wi_k * A.nu[(size_t)(3 + k) * ne + e];
        cHi -= wi_k * A.nu[(size_t)(6 + k) * ne + e];
        cGx += wx_k * A.nu[(size_t)(3 + k) * ne + ex];
        cHx += wx_k * A.nu[(size_t)(6 + k) * ne + ex];
      }
      double F0 = 0.0;
      const bool one_dry = wi == 0 || wx == 0;
      if (one_dry) F0 = llf_mass(ta, tb, nx, ny, P.g);
      if (!(one_dry && fabs(F0) > 1.0e-8)) {
        const double c[3] = {cF, cGi + cGx, cHi + cHx};
        llf_vjp(ta, tb, nx, ny, P.g, c, da, db);
      } else {  // internal_edge_hydro.F:212-302 with the forward's choice
        const bool in_dry = wi == 0;
        const bool refl = in_dry ? F0 > 0.0 : F0 < 0.0;
        if (refl) {
          // the wet side's state on both sides, its momentum reflected on the dry side
          const double* w = in_dry ? tb : ta;
          double rx, ry;
          reflect(nx, ny, w[1], w[2], rx, ry);
          const double wr[4] = {w[0], rx, ry, w[3]};
          const double c[3] = {cF, in_dry ? cGx : cGi, in_dry ? cHx : cHi};
          double dra[4], drb[4];
          llf_vjp(in_dry ? wr : ta, in_dry ? tb : wr, nx, ny, P.g, c, dra, drb);
          double* dw = in_dry ? db : da;
          const double* dref = in_dry ? dra : drb;
          const double* dself = in_dry ? drb : dra;
          dw[0] += dself[0] + dref[0];
          dw[3] += dself[3] + dref[3];
          dw[1] += dself[1];
          dw[2] += dself[2];
          reflect_t(nx, ny, dref[1], dref[2], dw[1], dw[2]);
        } else {
          // F and the wet side's momentum flux from the flux at G; the dry
          // side's momentum flux re-evaluated with G = 0
          const double cf[3] = {cF, in_dry ? cGx : cGi, in_dry ? cHx : cHi};
          const double cr[3] = {0.0, in_dry ? cGi : cGx, in_dry ? cHi : cHx};
          double d1[4], d2[4], d3[4], d4[4];
          llf_vjp(ta, tb, nx, ny, P.g, cf, d1, d2);
          llf_vjp(ta, tb, nx, ny, 0.0, cr, d3, d4);
          for (int k = 0; k < 4; ++k) { da[k] = d1[k] + d3[k]; db[k] = d2[k] + d4[k]; }
        }
      }
    }
    for (int k = 0; k < 4; ++k) { oi[k] = da[k]; ox[k] = db[k]; }
    return;
  }
  // land or ocean (other kinds are rejected before launch); a dry element
  // takes no boundary flux
  if (A.wd[e] == 0) {
    double* o = A.eb + (size_t)e * 36 + (3 * l + I) * 4;
    for (int k = 0; k < 4; ++k) o[k] = 0.0;
    return;
  }
  double q[9], hb[3];
  for (int c = 0; c < 9; ++c) q[c] = A.q[(size_t)c * ne + e];
  for (int k = 0; k < 3; ++k) hb[k] = m.hb[(size_t)k * ne + e];
  const int list = m.link[(size_t)l * ne + e];
  const double tx = -ny, ty = nx, den = 1.0 / (nx * ty - ny * tx);
  double ta[4], tb[4], c[3], da[4], db[4];
  trace(q, hb, l, I, ta);
  tb[0] = ta[0]; tb[1] = ta[1]; tb[2] = ta[2]; tb[3] = ta[3];
  bool fixed = false;
  if (kind == kOcean) {
    double zsum = 0.0;
    for (int f = 0; f < m.nbfr; ++f) {
      const double* zg = A.ocean_zg + ((size_t)f * m.needs + list) * 2;
      zsum = zsum + (0.5 * (zg[0] + zg[1]) + 0.5 * (zg[1] - zg[0]) * cB.xegp[I]);
    }
    if (zsum * P.ifnlfa + ta[3] <= 0) { zsum = fabs(ta[3]) + P.h0; fixed = true; }
    tb[0] = zsum;
  } else {
    const double qn = ta[1] * nx + ta[2] * ny, qt = ta[1] * tx + ta[2] * ty;
    tb[1] = (ty * (-qn) - ny * qt) * den;
    tb[2] = (-tx * (-qn) + nx * qt) * den;
  }
  const double jac = eg(EGeo::kXlen + l, e) / eg(EGeo::kAreas, e);  // XLEN/AREAS of the edge weights
  double wk[3];
  for (int k = 0; k < 3; ++k) wk[k] = 2.0 * cB.m_inv[k] * jac * cB.phi_edge[l][I][k] * cB.wegp[I];
  for (int v = 0; v < 3; ++v) {
    double cv = 0.0;
    for (int k = 0; k < 3; ++k) cv -= wk[k] * A.nu[(size_t)(3 * v + k) * ne + e];
    c[v] = cv;
  }
  llf_vjp(ta, tb, nx, ny, P.g, c, da, db);
  da[3] += db[3];  // the ghost keeps the in side's HB
  if (kind == kOcean) {
    if (fixed) da[3] += (ta[3] >= 0.0 ? 1.0 : -1.0) * db[0];
    da[1] += db[1];
    da[2] += db[2];
  } else {
    da[0] += db[0];
    // (xx, yx) = M (xi, yi): M^T applied to (dxx, dyx)
    const double dqne = (ty * db[1] - tx * db[2]) * den, dqte = (-ny * db[1] + nx * db[2]) * den;
    const double dqn = -dqne, dqt = dqte;
    da[1] += nx * dqn + tx * dqt;
    da[2] += ny * dqn + ty * dqt;
  }
  double* o = A.eb + (size_t)e * 36 + (3 * l + I) * 4;
  for (int k = 0; k < 4; ++k) o[k] = da[k];
}

// Element part: the volume terms' reverse mode at the three area points and
// the gather of the element's 36 edge-point trace cotangents through the
// basis; adds to lam, g_hb and g_n.
__global__ void __launch_bounds__(128, 5) elem_vjp(const __grid_constant__ AdjArgs A) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const MeshView& m = A.m;
  const int ne = m.ne;
  if (e >= ne) return;
  double q[9], hb[3], nu[9], lam9[9], ghb[3] = {0, 0, 0}, gn = 0.0;
  for (int c = 0; c < 9; ++c) {
    q[c] = A.q[(size_t)c * ne + e];
    nu[c] = A.nu[(size_t)c * ne + e];
    lam9[c] = 0.0;
  }
  for (int k = 0; k < 3; ++k) hb[k] = m.hb[(size_t)k * ne + e];
  auto eg = [&](int r, int el) { return m.egeo[(size_t)r * ne + el]; };
  const double geo[4] = {eg(EGeo::kDrdx, e), eg(EGeo::kDsdx, e), eg(EGeo::kDrdy, e), eg(EGeo::kDsdy, e)};
  const double nbar = m.manning ? eg(EGeo::kNbar, e) : 0.0;
  const int nvol = A.wd[e] != 0 ? 3 : 0;  // a dry element has no volume terms
  for (int i = 0; i < nvol; ++i) {
    double dv[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 1; k < 3; ++k) {
      const double dpx = cB.drphi[k][i] * geo[0] + cB.dsphi[k][i] * geo[1];
      const double dpy = cB.drphi[k][i] * geo[2] + cB.dsphi[k][i] * geo[3];
      const double xf = cB.mw[k][i] * dpx, yf = cB.mw[k][i] * dpy;
      dv[0] += xf * nu[k];     dv[1] += yf * nu[k];
      dv[2] += xf * nu[3 + k]; dv[3] += yf * nu[3 + k];
      dv[4] += xf * nu[6 + k]; dv[5] += yf * nu[6 + k];
    }
    for (int k = 0; k < 3; ++k) {
      dv[6] += cB.srfac[k][i] * nu[3 + k];
      dv[7] += cB.srfac[k][i] * nu[6 + k];
    }
    volume_vjp(A, e, i, q, hb, geo, nbar, dv, lam9, ghb, gn);
  }
  const double2* eb = reinterpret_cast<const double2*>(A.eb + (size_t)e * 36);
  for (int l = 0; l < 3; ++l)
    for (int gp = 0; gp < 3; ++gp) {
      const double2 a = eb[(3 * l + gp) * 2], b = eb[(3 * l + gp) * 2 + 1];
      for (int k = 0; k < 3; ++k) {
        const double p = cB.phi_edge[l][gp][k];
        lam9[k] += p * a.x;
        lam9[3 + k] += p * a.y;
        lam9[6 + k] += p * b.x;
        ghb[k] += p * b.y;
      }
    }
  for (int c = 0; c < 9; ++c) A.lam[(size_t)c * ne + e] += lam9[c];
  for (int k = 0; k < 3; ++k) A.g_hb[(size_t)k * ne + e] += ghb[k];
  if (A.g_n) A.g_n[e] += gn;
}

// ---- slope limiter 5 with frozen branches (slopelimiter.F:3259-3781) ----
// The forward limiter maps the stage kernel's output q (pre-limiter) to the
// stage state: per element and variable, vertex values clamped to the node
// min / max of the element means over each node's star, three
// mean-preserving redistribution sweeps, modes 2-3 rebuilt (mode 1 kept).
// With its decisions frozen (which clamp, the sweep signs, the counts of
// positive differences, which of the two limits each reduction takes) it is
// linear in q and in the node bounds; the bounds are the means of the first
// star element that attains them.

// Node min / max of the element means (as node_minmax) and the first star
// element attaining each: arg[(2 var + {0 min, 1 max}) * NP + n].
__global__ void node_arg(const MeshView m, const double* __restrict__ q, double* __restrict__ mm,
                         int* __restrict__ arg) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.np) return;
  const int ne = m.ne, np = m.np;
  for (int var = 0; var < 3; ++var) {
    double vmin = 99999., vmax = -99999.;
    int amin = -1, amax = -1;
    for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
      const int e = m.star[p];
      const double t = q[(size_t)(3 * var) * ne + e];
      if (t < vmin) { vmin = t; amin = e; }
      if (t > vmax) { vmax = t; amax = e; }
    }
    mm[(size_t)(2 * var) * np + n] = vmin;
    mm[(size_t)(2 * var + 1) * np + n] = vmax;
    arg[(size_t)(2 * var) * np + n] = amin;
    arg[(size_t)(2 * var + 1) * np + n] = amax;
  }
}

__device__ __forceinline__ double div_count(double x, int kdp) {
  if (kdp <= 1) return x;
  if (kdp == 2) return x * 0.5;
  return x / 3.0;
}

// Reverse mode of WETDRY (wetdry.F:61-548) for element e with its branches
// frozen, at its input q (the limited state) and input flag wd_in: lam from
// the cotangent of WETDRY's output to that of its input; ghb1 / ghb2 += the
// terms of the flattening (ZE modes 2-3 set to -HB modes 2-3).  The nodal
// depths DP are constants here.
__device__ void wetdry_vjp(const MeshView& m, const Physics& ph, int e, int wd_in, const double q[9], double lam[9],
                           double& ghb1, double& ghb2) {
  const int ne = m.ne;
  const double H0 = ph.h0, ZERO = 1.0e-6, c13 = 1.0 / 3.0, c16 = 1.0 / 6.0;
  double dpn[3];
  for (int v = 0; v < 3; ++v) dpn[v] = m.dp[m.nm[(size_t)v * ne + e]];
  const double dpe_min = fmin(fmin(dpn[0], dpn[1]), dpn[2]);
  int ndry = 0, hmax_i = 0;
  double hmax = ZERO, ht[3], zn[3];
  for (int v = 0; v < 3; ++v) {
    zn[v] = q[0] + cB.phi_corner[v][1] * q[1] + cB.phi_corner[v][2] * q[2];
    ht[v] = dpn[v] + zn[v];
    if (ht[v] > hmax) { hmax_i = v; hmax = ht[v]; }
    if (ht[v] <= H0 + ZERO) ++ndry;
  }
  const double dp_avg = c13 * (dpn[0] + dpn[1] + dpn[2]);
  if (ndry == 0) {
    if (wd_in == 1) return;  // unchanged
    // the element check alone: momentum zeroed if the highest vertex is too low
    if (!(zn[hmax_i] > (-dpe_min + H0)))
      for (int c = 3; c < 9; ++c) lam[c] = 0.0;
    return;
  }
  const double ht_avg = q[0] + dp_avg;
  if (ndry == 3 || ht_avg <= H0 + ZERO) {  // flatten: ZE1 = ht_avg - dp_avg, ZE2,3 = -HB2,3, no momentum
    ghb1 -= lam[1];
    ghb2 -= lam[2];
    if (ht_avg < ZERO) lam[0] = 0.0;
    lam[1] = 0.0;
    lam[2] = 0.0;
    for (int c = 3; c < 9; ++c) lam[c] = 0.0;
    return;
  }
  // case 3B: replay, recording the branches
  int l2h[3] = {0, 1, 2};
  for (int k1 = 0; k1 < 3; ++k1)
    for (int k2 = k1; k2 < 3; ++k2)
      if (ht[l2h[k1]] > ht[l2h[k2]]) { const int t = l2h[k1]; l2h[k1] = l2h[k2]; l2h[k2] = t; }
  double dh[3];
  const bool b0 = H0 >= ht[l2h[0]];
  dh[l2h[0]] = fmax(H0, ht[l2h[0]]) - ht[l2h[0]];
  const bool b1 = H0 >= ht[l2h[1]] - 0.5 * dh[l2h[0]];
  dh[l2h[1]] = fmax(H0, ht[l2h[1]] - 0.5 * dh[l2h[0]]) - ht[l2h[1]];
  dh[l2h[2]] = -dh[l2h[0]] - dh[l2h[1]];
  int nd2 = 0;
  double hmax2 = 0.0, hh[3];
  bool dry[3];
  for (int v = 0; v < 3; ++v) {
    hh[v] = ht[v] + dh[v];
    if (hh[v] > hmax2) { hmax_i = v; hmax2 = hh[v]; }
    dry[v] = hh[v] <= H0 + 1.0e-10;
    if (dry[v]) ++nd2;
  }
  const bool keep_mom = (hh[hmax_i] - dpn[hmax_i]) > (-dpe_min + H0);
  // reverse: momentum (rebuilt from wet vertices plus the dry vertices' share)
  double din[9] = {lam[0], 0, 0, 0, 0, 0, 0, 0, 0};
  if (keep_mom && nd2 < 3) {
    for (int w = 0; w < 2; ++w) {  // QX modes 3..5, QY modes 6..8
      const double* dq = lam + 3 + 3 * w;
      const double dqh[3] = {c13 * dq[0] - c16 * dq[1] - 0.5 * dq[2], c13 * dq[0] - c16 * dq[1] + 0.5 * dq[2],
                             c13 * dq[0] + c13 * dq[1]};
      double ds = 0.0;
      for (int v = 0; v < 3; ++v)
        if (!dry[v]) ds += dqh[v];
      for (int v = 0; v < 3; ++v) {
        const double dn = dry[v] ? ds / (3.0 - (double)nd2) : dqh[v];
        din[3 + 3 * w] += dn;
        din[4 + 3 * w] += cB.phi_corner[v][1] * dn;
        din[5 + 3 * w] += cB.phi_corner[v][2] * dn;
      }
    }
  }
  // elevation: ZE2,3 from the vertex elevations hh - DP, ZE1 kept
  const double dzh[3] = {-c16 * lam[1] - 0.5 * lam[2], -c16 * lam[1] + 0.5 * lam[2], c13 * lam[1]};
  double dht[3], ddh[3];
  for (int v = 0; v < 3; ++v) { dht[v] = dzh[v]; ddh[v] = dzh[v]; }
  ddh[l2h[0]] -= ddh[l2h[2]];
  ddh[l2h[1]] -= ddh[l2h[2]];
  if (b1) dht[l2h[1]] -= ddh[l2h[1]];
  else ddh[l2h[0]] += -0.5 * ddh[l2h[1]];
  if (b0) dht[l2h[0]] -= ddh[l2h[0]];
  for (int v = 0; v < 3; ++v) {
    din[0] += dht[v];
    din[1] += cB.phi_corner[v][1] * dht[v];
    din[2] += cB.phi_corner[v][2] * dht[v];
  }
  for (int c = 0; c < 9; ++c) lam[c] = din[c];
}

// Per element: replay of the limiter (slopeflag) and WETDRY (wetdry) on the
// pre-limiter state q, then their reverse modes.  lam (in place): the
// cotangent of the stage state on entry, of the pre-limiter state on exit
// (without the bound terms); lb[e*18 + (var*3 + a)*2 + {0 min, 1 max}]: the
// cotangent of vertex a's bounds; g_hb += WETDRY's HB terms.
__global__ void __launch_bounds__(128, 5) limit_vjp(const MeshView m, const Physics ph, int slopeflag, int wetdry,
                                                 const int* __restrict__ wd, const double* __restrict__ q,
                                                 const double* __restrict__ mm, double* __restrict__ lam,
                                                 double* __restrict__ lb, double* __restrict__ g_hb) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = m.ne, np = m.np;
  if (e >= ne) return;
  int nd[3];
  for (int v = 0; v < 3; ++v) nd[v] = m.nm[(size_t)v * ne + e];
  double ql[9], l9[9];
  for (int c = 0; c < 9; ++c) {
    ql[c] = q[(size_t)c * ne + e];
    l9[c] = lam[(size_t)c * ne + e];
  }
  // limiter replay, keeping its decisions
  int clamp[3][3];
  double sgn[3][3];
  bool pos[3][3][3], to_max[3][3][3];
  int kd[3][3][3];
  if (slopeflag != 0) {
    for (int var = 0; var < 3; ++var) {
      const double* z = ql + 3 * var;
      double vmin[3], vmax[3], vx[3];
      for (int a = 0; a < 3; ++a) {
        vmin[a] = mm[(size_t)(2 * var) * np + nd[a]];
        vmax[a] = mm[(size_t)(2 * var + 1) * np + nd[a]];
        const double v = z[0] + cB.phi_corner[a][1] * z[1] + cB.phi_corner[a][2] * z[2];
        const double c1 = fmin(v, vmax[a]);
        vx[a] = fmax(c1, vmin[a]);
        clamp[var][a] = vx[a] != c1 ? 2 : (c1 != v ? 1 : 0);
      }
      for (int w = 0; w < 3; ++w) {
        const double sumloc = (vx[0] + vx[1] + vx[2]) / 3.0;
        double sumdif = (sumloc - z[0]) * 3.0;
        const double s = copysign(1.0, sumdif);
        sgn[var][w] = s;
        double dif[3];
        for (int a = 0; a < 3; ++a) dif[a] = (vx[a] - z[0]) * s;
        int kdp = (dif[0] > 0) + (dif[1] > 0) + (dif[2] > 0);
        for (int k = 0; k < 3; ++k) {
          double redfac = 0.0;
          pos[var][w][k] = dif[k] > 0;
          kd[var][w][k] = kdp;
          if (pos[var][w][k]) {
            redfac = div_count(sumdif * s, kdp);
            kdp = kdp - 1;
          }
          const double redmax = s > 0 ? vx[k] - vmin[k] : vmax[k] - vx[k];
          to_max[var][w][k] = !(redfac <= redmax);
          redfac = fmin(redfac, redmax);
          sumdif = sumdif - redfac * s;
          vx[k] = vx[k] - redfac * s;
        }
      }
      ql[3 * var + 1] = -(1.0 / 6.0 * (vx[0] + vx[1])) + 1.0 / 3.0 * vx[2];
      ql[3 * var + 2] = -(.5 * vx[0]) + .5 * vx[1];
    }
  }
  if (wetdry != 0) {
    double g1 = 0.0, g2 = 0.0;
    wetdry_vjp(m, ph, e, wd[e], ql, l9, g1, g2);
    g_hb[(size_t)ne + e] += g1;
    g_hb[(size_t)2 * ne + e] += g2;
  }
  if (slopeflag != 0) {
    for (int var = 0; var < 3; ++var) {
      const double l0 = l9[3 * var], l1 = l9[3 * var + 1], l2 = l9[3 * var + 2];
      double dz[3] = {l0, 0.0, 0.0}, dvx[3], dmin[3] = {0, 0, 0}, dmax[3] = {0, 0, 0};
      dvx[0] = -(1.0 / 6.0) * l1 - 0.5 * l2;
      dvx[1] = -(1.0 / 6.0) * l1 + 0.5 * l2;
      dvx[2] = (1.0 / 3.0) * l1;
      for (int w = 2; w >= 0; --w) {
        const double s = sgn[var][w];
        double dsum = 0.0;  // cotangent of sumdif along the sweep
        for (int k = 2; k >= 0; --k) {
          const double dred = -s * dsum - s * dvx[k];
          if (to_max[var][w][k]) {
            if (s > 0) { dvx[k] += dred; dmin[k] -= dred; }
            else { dmax[k] += dred; dvx[k] -= dred; }
          } else if (pos[var][w][k]) {
            const int d = kd[var][w][k];
            dsum += (d <= 1 ? 1.0 : (d == 2 ? 0.5 : 1.0 / 3.0)) * s * dred;
          }
        }
        for (int a = 0; a < 3; ++a) dvx[a] += dsum;  // sumdif = vx0 + vx1 + vx2 - 3 z0 at the sweep's start
        dz[0] -= 3.0 * dsum;
      }
      for (int a = 0; a < 3; ++a) {
        if (clamp[var][a] == 1) dmax[a] += dvx[a];
        else if (clamp[var][a] == 2) dmin[a] += dvx[a];
        else {
          dz[0] += dvx[a];
          dz[1] += cB.phi_corner[a][1] * dvx[a];
          dz[2] += cB.phi_corner[a][2] * dvx[a];
        }
        lb[(size_t)e * 18 + (var * 3 + a) * 2] = dmin[a];
        lb[(size_t)e * 18 + (var * 3 + a) * 2 + 1] = dmax[a];
      }
      l9[3 * var] = dz[0];
      l9[3 * var + 1] = dz[1];
      l9[3 * var + 2] = dz[2];
    }
  }
  for (int c = 0; c < 9; ++c) lam[(size_t)c * ne + e] = l9[c];
}

// Per node: the cotangents of its bounds, summed over its star in star order.
__global__ void node_bound_gather(const MeshView m, const double* __restrict__ lb, double* __restrict__ nb) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= m.np) return;
  const int ne = m.ne, np = m.np;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int p = m.star_ptr[n]; p < m.star_ptr[n + 1]; ++p) {
    const int e = m.star[p];
    const int a = m.nm[e] == n ? 0 : (m.nm[(size_t)ne + e] == n ? 1 : 2);
    for (int var = 0; var < 3; ++var) {
      acc[2 * var] += lb[(size_t)e * 18 + (var * 3 + a) * 2];
      acc[2 * var + 1] += lb[(size_t)e * 18 + (var * 3 + a) * 2 + 1];
    }
  }
  for (int r = 0; r < 6; ++r) nb[(size_t)r * np + n] = acc[r];
}

// Per element: the node-bound cotangents of the nodes whose min / max it
// attains, added to its mean (mode 1) of that variable.
__global__ void elem_bound_scatter(const MeshView m, const int* __restrict__ arg, const double* __restrict__ nb,
                                   double* __restrict__ lam) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ne = m.ne, np = m.np;
  if (e >= ne) return;
  double add[3] = {0, 0, 0};
  for (int v = 0; v < 3; ++v) {
    const int n = m.nm[(size_t)v * ne + e];
    if (v == 1 && n == m.nm[e]) continue;  // a node listed twice counts once
    if (v == 2 && (n == m.nm[e] || n == m.nm[(size_t)ne + e])) continue;
    for (int r = 0; r < 6; ++r)
      if (arg[(size_t)r * np + n] == e) add[r / 2] += nb[(size_t)r * np + n];
  }
  for (int var = 0; var < 3; ++var) lam[(size_t)(3 * var) * ne + e] += add[var];
}

void launch_limit_vjp(const MeshView& m, const Physics& ph, int slopeflag, int wetdry, const int* wd,
                      const double* qpre, double* mm, int* arg, double* lam, double* lb, double* nb, double* g_hb,
                      cudaStream_t s) {
  const unsigned gn = (unsigned)((m.np + 127) / 128), ge = (unsigned)((m.ne + 127) / 128);
  if (slopeflag != 0) node_arg<<<gn, 128, 0, s>>>(m, qpre, mm, arg);
  limit_vjp<<<ge, 128, 0, s>>>(m, ph, slopeflag, wetdry, wd, qpre, mm, lam, lb, g_hb);
  if (slopeflag != 0) {
    node_bound_gather<<<gn, 128, 0, s>>>(m, lb, nb);
    elem_bound_scatter<<<ge, 128, 0, s>>>(m, arg, nb, lam);
  }
}

// lam_I += a_I lam_j, nu_I += b_I lam_j for I < n, over all 9*NE values
// (first: lam_I = a_I lam_j, nu_I = b_I lam_j)
__global__ void ssp_adj(const __grid_constant__ SspAdjArgs A) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.len) return;
  const double l = A.lam_j[i];
  if (A.first) {
    for (int I = 0; I < A.n; ++I) {
      A.lam[I][i] = A.a[I] != 0.0 ? A.a[I] * l : 0.0;
      A.nu[I][i] = A.b[I] != 0.0 ? A.b[I] * l : 0.0;
    }
    return;
  }
  for (int I = 0; I < A.n; ++I) {
    if (A.a[I] != 0.0) A.lam[I][i] += A.a[I] * l;
    if (A.b[I] != 0.0) A.nu[I][i] += A.b[I] * l;
  }
}

__global__ void gauge_eval(const double* __restrict__ q, int ne, const int* __restrict__ elem,
                           const double* __restrict__ phi, int ng, double* __restrict__ eta) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ng) return;
  const int e = elem[g];
  eta[g] = phi[3 * g] * q[e] + phi[3 * g + 1] * q[(size_t)ne + e] + phi[3 * g + 2] * q[(size_t)2 * ne + e];
}

// Misfit seed: one thread per distinct gauge element, which adds its gauges
// in input order (deterministic where gauges share an element).
__global__ void gauge_seed(double* lam, int ne, const int* __restrict__ gel, const int* __restrict__ gptr,
                           const int* __restrict__ ggauge, const double* __restrict__ phi,
                           const double* __restrict__ w, int ngroup) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ngroup) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = gptr[t]; i < gptr[t + 1]; ++i) {
    const int g = ggauge[i];
    a0 += phi[3 * g] * w[g];
    a1 += phi[3 * g + 1] * w[g];
    a2 += phi[3 * g + 2] * w[g];
  }
  const int e = gel[t];
  lam[e] += a0;
  lam[(size_t)ne + e] += a1;
  lam[(size_t)2 * ne + e] += a2;
}

void launch_rhs_vjp(const AdjArgs& a, cudaStream_t s) {
  if (a.m.ne <= 0) return;
  if (a.nedge > 0) edge_vjp<<<(unsigned)((3LL * a.nedge + 255) / 256), 256, 0, s>>>(a);
  elem_vjp<<<(unsigned)((a.m.ne + 127) / 128), 128, 0, s>>>(a);
}

void launch_ssp_adj(const SspAdjArgs& a, cudaStream_t s) {
  if (a.len <= 0 || a.n <= 0) return;
  ssp_adj<<<(unsigned)((a.len + 255) / 256), 256, 0, s>>>(a);
}

void launch_gauge_eval(const double* q, int ne, const int* elem, const double* phi, int ng, double* eta,
                       cudaStream_t s) {
  if (ng <= 0) return;
  gauge_eval<<<(unsigned)((ng + 127) / 128), 128, 0, s>>>(q, ne, elem, phi, ng, eta);
}

void launch_gauge_seed(double* lam, int ne, const int* gel, const int* gptr, const int* ggauge, const double* phi,
                       const double* w, int ngroup, cudaStream_t s) {
  if (ngroup <= 0) return;
  gauge_seed<<<(unsigned)((ngroup + 127) / 128), 128, 0, s>>>(lam, ne, gel, gptr, ggauge, phi, w, ngroup);
}

}  // namespace adj
}  // namespace dgswem
