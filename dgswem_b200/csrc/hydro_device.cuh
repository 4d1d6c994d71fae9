// hydro_device.cuh -- device data layout and kernels of the p=1 DG hydro step.
//
// Layout in HBM (NE elements, NP nodes, all structure-of-arrays so a warp's
// 32 consecutive elements make one coalesced transaction per field).
// Elements are in the device order (a Morton curve of the centroids, built
// at create; perm/inv map it to the input numbering):
//   state   q[c*NE + e], c = 3*var + k  (var: 0 zeta, 1 qx, 2 qy; k: mode)
//   nm[v*NE + e]       0-based vertex node ids
//   link[l*NE + e]     across local edge l: neighbour element (interior edge)
//                      or index into the boundary list of that edge's kind
//   einfo[e]           packed edge kinds, processing order, orientation bits
//   hb[k*NE + e]       bathymetry modes HB(k,e)
//   stage tile plan    per tile of consecutive elements (TileShape): its edge tasks
//                      (uint2 each, interior edges first, then boundary kinds)
//                      and its halo (out-of-tile neighbours, global ids);
//                      eslot[e] names the task of each local edge
// Geometry (areas, Jacobian, edge lengths and normals) is recomputed from the
// nodal coordinates each stage, with the reference's formulas, instead of
// streaming the reference's per-element tables (XFAC/YFAC/SRFAC/BATHED: ~100
// doubles per element).
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

namespace dgswem {

constexpr int kMaxStages = 8;

enum EdgeKind : unsigned {
  kInterior = 0,
  kOcean = 1,      // ocean_edge_hydro.F
  kLand = 2,       // land_edge_hydro.F
  kFlow = 3,       // flow_edge_hydro.F
  kRadiation = 4,  // radiation_edge_hydro.F
  kIBarrier = 5,   // ibarrier_edge_hydro.F
  kEBarrier = 6,   // ebarrier_edge_hydro.F
  kNone = 7        // boundary edge in no list: the reference skips it
};

// einfo bit fields
__host__ __device__ inline unsigned ei_kind(unsigned info, int l) { return (info >> (3 * l)) & 7u; }
__host__ __device__ inline unsigned ei_flag(unsigned info, int l) { return (info >> (9 + l)) & 1u; }
__host__ __device__ inline unsigned ei_nled(unsigned info, int l) { return (info >> (12 + 2 * l)) & 3u; }
__host__ __device__ inline unsigned ei_order(unsigned info, int s) { return (info >> (18 + 2 * s)) & 3u; }

// p=1 basis tables (orthogonal_basis_v1.F, prep_DG.F:648-870), Lobatto edge
// rule (quad_rules_general.F) and 3-point area rule (quadrature_v1.F:255-260).
// Built in FP64 on the host; the mixed-precision kernels also keep an FP32
// copy for their FP32 arithmetic.
template <class T>
struct BasisT {
  T phi_edge[3][3][3];  // [led][point][mode]
  T edgeq[3][3][3];     // 2*M_INV*PHI_EDGE*WEGP
  T phi_area[3][3];     // [mode][point]
  T drphi[3][3], dsphi[3][3];
  T phi_corner[3][3];   // [vertex][mode]
  T psi[3][3];          // [vertex][area point] linear nodal basis
  T m_inv[3], wagp[3], wegp[3], xegp[3];
  T mw[3][3];           // [mode][point] M_INV*WAGP
  T srfac[3][3];        // [mode][point] M_INV*WAGP*PHI_AREA (SRFAC without the area)
};
using BasisP1 = BasisT<double>;
static_assert(sizeof(BasisT<float>) * 2 == sizeof(BasisT<double>), "basis tables are plain arrays");

struct MeshView {
  int ne, np;
  const double* __restrict__ x;
  const double* __restrict__ y;
  const double* __restrict__ dp;        // nodal depth
  const int* __restrict__ nm;
  const int* __restrict__ link;
  const unsigned* __restrict__ einfo;
  const double* __restrict__ hb;
  const double* __restrict__ egeo;      // [r*NE + e] element geometry rows (EGeo)
  const float* __restrict__ egeof;      // the same rows in FP32 (mixed-precision handles), or null
  const double* __restrict__ cori;      // per element, or null (uniform)
  const double* __restrict__ fric;      // per element, or null (uniform)
  const double* __restrict__ manning;   // nodal, or null
  const double* __restrict__ sfac_area; // [i*NE+e] (ics=2) or null
  const double* __restrict__ sfac_edge; // [(l*3+i)*NE+e] (ics=2) or null
  const int* __restrict__ star_ptr;     // node -> element star (CSR)
  const int* __restrict__ star;
  const int* __restrict__ node_perm;    // device node -> input node
  // boundary lists
  int needs, nfeds, nebseg, nibseg, nbfr, nffr;
  const double* __restrict__ emo_dg;    // EMO_DG(NBFR,NEEDS,2)
  const double* __restrict__ efa_dg;
  const double* __restrict__ qnam_dg;   // QNAM_DG(NFFR,NFEDS,2)
  const double* __restrict__ qnph_dg;
  const double* __restrict__ ebht;
  const double* __restrict__ ebcfsp;
  const int* __restrict__ ib_elem;      // [2*L + side] element of back/front edge
  const int* __restrict__ ib_led;       // [2*L + side] local edge
  const double* __restrict__ ibht;
  const double* __restrict__ ibcfsb;
  const double* __restrict__ ibcfsp;
  // stage tile plan (built at create from the edge graph, rebuilt when the
  // tile shape changes)
  int max_halo, max_tasks;                // largest halo / task list of a tile
  const int* __restrict__ tile_elem_ptr;  // [ntile+1] first element of each tile
  const int* __restrict__ tile_task_ptr;  // [ntile+1] offsets into tile_tasks
  const uint2* __restrict__ tile_tasks;   // TaskBits word, list index
  const int* __restrict__ tile_halo_ptr;  // [ntile+1] offsets into tile_halo
  const int* __restrict__ tile_halo;      // global element ids, ascending
  const unsigned* __restrict__ eslot;     // task of local edge l: bits 10l..10l+9
};

// Stage tile shapes the stage kernel is compiled in: a tile of up to `tile`
// consecutive elements and `threads` edge tasks per block of `threads`.
// Every shape gives the same results bit for bit (each edge point's flux is
// evaluated in the reference's in/ex orientation whichever tile evaluates
// it, and each element's sums keep the reference's order); the autotuner
// (dgswem_cuda_autotune) picks the fastest for a mesh.  `tile` is a multiple
// of 32 (phase 3 keeps an area point per warp) and `threads` a multiple of
// `tile` above it (phase 1 copies rows by whole groups of `tile` threads).
struct TileShape {
  int tile, threads;
};
constexpr int kNumTileShapes = 4;
constexpr TileShape kTileShapes[kNumTileShapes] = {{128, 384}, {64, 192}, {64, 256}, {256, 768}};
constexpr int kDefaultTileShape = 0;
// Block sizes of the limiter / WETDRY element kernel (limit_wetdry), each
// compiled for 1024 resident threads per SM except the last (768: more
// registers per thread)
constexpr int kNumLimitShapes = 3;
constexpr int kLimitBlocks[kNumLimitShapes] = {256, 128, 256};
constexpr int kLimitMinBlocks[kNumLimitShapes] = {4, 8, 3};
constexpr int kDefaultLimitShape = 0;
constexpr unsigned kNoTask = 1023u;
constexpr int kMaxTileSlots = 512;  // tile + halo rows addressable by a task word's 9-bit slots

// Task word of the tile plan.  Slots index the tile's shared-memory element
// rows: 0..tile-1 the tile's own elements, tile+j halo element j.
struct TaskBits {
  static constexpr int kKind = 0;     // 3 bits, EdgeKind
  static constexpr int kLedIn = 3;    // 2 bits, local edge of the in side
  static constexpr int kLedEx = 5;    // 2 bits, local edge of the ex side
  static constexpr int kFlip = 7;     // the in side is a halo element: normal = -(ex side's normal)
  static constexpr int kInSlot = 8;   // 9 bits
  static constexpr int kExSlot = 17;  // 9 bits
};

// Rows of the element geometry table, computed once at create from the
// nodal coordinates with the reference's formulas (read_input.F:1406 AREAS,
// calc_normal.F:41-48 XLEN and normals on the counter-clockwise local edges,
// rhs_dg_hydro.F's DRDX/DSDX/DRDY/DSDY from the area and the coordinate
// differences, XLEN/AREAS of internal_edge_hydro.F) and the element mean of
// the nodal Manning n.  The stage kernel copies the first kSmemRows (with
// Manning n) into shared memory; AREAS and XLEN, used only by boundary
// edges, are read from the table.
struct EGeo {
  static constexpr int kNx = 0, kNy = 3, kDrdx = 6, kDsdx = 7, kDrdy = 8, kDsdy = 9, kEdfac = 10, kNbar = 13;
  static constexpr int kAreas = 14, kXlen = 15, kRows = 18;
  static constexpr int kSmemRows = 14;
};

// Dynamic shared memory of the stage kernel (byte offsets).  Per-element
// rows of geo: the first EGeo::kSmemRows rows of the table, then the hybrid
// friction factor.
struct SGeo {
  static constexpr int kHyb = EGeo::kSmemRows;
};
constexpr int kGeoRows = EGeo::kSmemRows + 1;
constexpr int kVolRows = 8;  // per area point: fx fy gx gy hx hy sx sy
// doubles per element slot of the shared state: 12 modal values and a pad,
// a 112-byte stride that keeps 16-byte loads by 8 consecutive slots free of
// bank conflicts
constexpr unsigned kQStride = 14;
// floats per element slot of the FP32 copy of the shared state (mixed
// precision): the 12 modal values, three 16-byte loads, a 48-byte stride
// that is conflict-free for 8 consecutive slots
constexpr unsigned kQfStride = 12;
struct StageLayout {
  unsigned qs, geo, qf, vol, res, wd, gid, tdry, info, tasks, bytes;
};
__host__ __device__ inline unsigned align16(unsigned x) { return (x + 15u) & ~15u; }
// tile: elements per tile of the shape; rb: bytes of the arithmetic type of
// the edge and volume terms (8: FP64 kernels; 4: mixed precision, which adds
// the FP32 slot copy qf)
__host__ __device__ inline StageLayout stage_layout(int tile, int max_halo, int max_tasks, unsigned rb) {
  StageLayout L;
  const unsigned nt = (unsigned)tile;
  const unsigned S = nt + (unsigned)max_halo;
  const unsigned T = (unsigned)max_tasks;
  L.qs = 0;  // the basis tables are read from constant memory
  // qs[S][kQStride]: ZE, QX, QY, HB modes (mixed: the tile's own slots only,
  // for the FP64 SSP combination; the edge and volume terms read qf)
  L.geo = L.qs + kQStride * (rb == 8u ? S : nt) * 8u;
  L.qf = L.geo + kGeoRows * nt * rb;           // geo[kGeoRows][tile] in the arithmetic type
  L.vol = L.qf + (rb == 8u ? 0u : kQfStride * S * 4u);  // qf[S][kQfStride] (mixed only)
  L.res = L.vol + kVolRows * 3u * nt * rb;     // vol[kVolRows][3][tile]
  // res[task][point][5]; the mixed variant first stages the halo's FP64
  // values there (12 doubles an element)
  const unsigned res_bytes = 15u * T * rb, stage_bytes = rb == 8u ? 0u : 96u * (unsigned)max_halo;
  L.wd = L.res + (res_bytes > stage_bytes ? res_bytes : stage_bytes);
  L.gid = align16(L.wd + S * 4u);              // wd[S]
  L.tdry = align16(L.gid + (unsigned)max_halo * 4u);
  L.info = align16(L.tdry + T * 4u);          // einfo, eslot of the tile's elements
  L.tasks = align16(L.info + 2u * nt * 4u);    // the tile's edge-task words (uint2)
  L.bytes = align16(L.tasks + T * 8u);
  return L;
}

struct Physics {
  double g, h0, dtdp, nleq, leq, nleqg, fg_l;
  double tau_cap;  // .9 * (1 / DTDP), the friction cap of rhs_dg_hydro.F
  double cori, fric, cf, hbreak, ftheta, fgamma;
  int iflinbf, ifhybf, ifnlfa, nws, rainfall, ics;
};

// Physics constants of the stage kernel's FP32 terms (mixed precision)
struct PhysF {
  float g, nleq, leq, nleqg, fg_l, tau_cap, cori, fric, cf;
};

struct StageArgs {
  MeshView m;
  Physics ph;
  PhysF pf;  // ph rounded to FP32
  int irk;                                  // 1-based stage
  const double* __restrict__ qin;           // state of stage irk (edges read it)
  double* qout;                             // state of stage irk+1
  const double* qhist[kMaxStages];          // state of stage I, I=1..irk
  const double* rhist[kMaxStages];          // RHS of stage I<irk (if needed)
  double* rout;                             // this stage's RHS, or null
  double a[kMaxStages], b[kMaxStages];      // ATVD(irk,I), BTVD(irk,I)*DT
  const int* __restrict__ wd;               // WDFLG (read)
  double timedg, rampdg;
  const double* __restrict__ ramp;          // RAMPDG of this stage in device memory (graph replays), or null: rampdg
  const double* __restrict__ ocean_zg;      // [(f*NEEDS + L)*2 + ipt] EMO*RFF*COS(ARGJ-EFA)
  const double* __restrict__ flow_qn;       // [(f*NFEDS + L)*3 + point] QNAM*RFF*COS(ARG)
  const double* __restrict__ wsx;           // nodal met forcing (already ramped), or null
  const double* __restrict__ wsy;
  const double* __restrict__ pr;
  double* ib_rhs;                           // [(2*seg + side)*9 + c] internal-barrier terms
  unsigned* err;                            // device error word
  // tiles of this launch: block b runs tile tile_list[tile_off + b], or
  // tile b when tile_list is null (all tiles)
  const int* __restrict__ tile_list;
  int tile_off;
};

struct LimitArgs {
  MeshView m;
  Physics ph;
  double* q;                 // stage output, limited / wet-dried in place
  double* minmax;            // [6*NP]: (min, max) pairs of ZE, QX, QY means per node
  int* wd;                   // WDFLG (read + write)
  int slopeflag, wetdry;
  int ne_act;                // elements limited / wet-dried: the owned ones (the first ne_act)
  unsigned* err;
};

// Kernel launchers, one set per compilation variant: `fast` lets the
// compiler contract a*b+c into FMA; `strict` (-fmad=false) keeps every
// product and sum separately rounded, the evaluation the FP64 oracle uses;
// `mixed` is `fast` with the stage kernel's edge and volume arithmetic in
// FP32 (state, SSP combination, limiter and wet/dry stay FP64).
#define DGSWEM_DECLARE_LAUNCHERS(NS)                                                           \
  namespace NS {                                                                               \
  void set_basis(const BasisP1& b);                                                            \
  void launch_stage(const StageArgs& a, bool nonlin, int shape, unsigned grid, size_t smem,       \
                    cudaStream_t s);                                                           \
  void launch_ibarrier(const StageArgs& a, bool nonlin, cudaStream_t s);                       \
  void launch_node_minmax(const LimitArgs& a, unsigned grid, cudaStream_t s);                  \
  void launch_limit_wetdry(const LimitArgs& a, int shape, cudaStream_t s);                      \
  void launch_modal2nodal(const MeshView& m, const double* q, const int* wd, double nleq,      \
                          double leq, double* eta2, double* uu2, double* vv2, int* nodecode,   \
                          unsigned grid, cudaStream_t s);                                      \
  void launch_fortran_to_soa(const double* f, double* q, int ne, int var, const int* perm,     \
                             unsigned grid, cudaStream_t s);                                   \
  void launch_soa_to_fortran(const double* q, double* f, int ne, int var, const int* inv,      \
                             unsigned grid, cudaStream_t s);                                   \
  void launch_gather_int(const int* src, int* dst, const int* idx, int n, unsigned grid,       \
                         cudaStream_t s);                                                      \
  void launch_halo(bool pack, double* q, int* wd, int ne, const int* idx, int n, int kind,     \
                   double* buf, cudaStream_t s);                                               \
  }

DGSWEM_DECLARE_LAUNCHERS(fast)
DGSWEM_DECLARE_LAUNCHERS(strict)
DGSWEM_DECLARE_LAUNCHERS(mixed)

// ---- p=2 (hydro_p2.cuh, kernels_p2_fast.cu / kernels_p2_strict.cu) --------
// Six modes per variable, the four-point Gauss-Lobatto edge rule and the
// six-point area rule (quadrature_v1.F); FP64, no wet/dry, no limiter.
constexpr int kP2Modes = 6, kP2Egp = 4, kP2Agp = 6;
template <class T>
struct BasisP2T {
  T phi_edge[3][kP2Egp][kP2Modes];  // [led][point][mode]
  T edgeq[3][kP2Egp][kP2Modes];     // 2*M_INV*PHI_EDGE*WEGP
  T phi_area[kP2Modes][kP2Agp];     // [mode][point]
  T drphi[kP2Modes][kP2Agp], dsphi[kP2Modes][kP2Agp];
  T phi_corner[3][kP2Modes];        // [vertex][mode]
  T psi[3][kP2Agp];                 // linear nodal basis at the area points
  T m_inv[kP2Modes], wagp[kP2Agp], wegp[kP2Egp], xegp[kP2Egp];
  T mw[kP2Modes][kP2Agp];           // M_INV*WAGP
  T srfac[kP2Modes][kP2Agp];        // M_INV*WAGP*PHI_AREA
};
using BasisP2 = BasisP2T<double>;
static_assert(sizeof(BasisP2T<float>) * 2 == sizeof(BasisP2), "p=2 basis tables are plain arrays");
struct P2Args {
  MeshView m;   // hb: six rows; egeo; einfo / link for the edge kinds and neighbours
  Physics ph;
  PhysF pf;     // ph rounded to FP32 (mixed precision)
  int irk;
  const double* __restrict__ qin;  // 18 rows (6*var + mode)
  double* qout;
  const double* qhist[kMaxStages];
  const double* rhist[kMaxStages];
  double* rout;
  double a[kMaxStages], b[kMaxStages];
  double rampdg;
  const double* __restrict__ ramp;  // RAMPDG in device memory (graph replays), or null: rampdg
  const double* __restrict__ ocean_zg;
  const double* __restrict__ wsx;
  const double* __restrict__ wsy;
  const double* __restrict__ pr;
  double* ef;                      // [((e*3 + led)*4 + point)*3 + c] edge-point fluxes F, G, H per side
                                   // (in the arithmetic type: FP32 in the mixed variant)
  const int* __restrict__ edges;   // (element, local edge): interior edges from the in side, land and ocean edges
  int nedge, ne_act;
  unsigned* err;
  int ntile;                       // tiles of the tile plan: > 0 runs the p=2 tile kernel (p2_tile)
};
#define DGSWEM_DECLARE_P2_LAUNCHERS(NS)                                                          \
  namespace NS {                                                                                 \
  void set_basis_p2(const BasisP2& b);                                                           \
  void launch_p2_stage(const P2Args& a, bool nonlin, cudaStream_t s);                            \
  void launch_p2_modal2nodal(const MeshView& m, const double* q, double nleq, double leq,         \
                             double* eta2, double* uu2, double* vv2, int* nodecode, cudaStream_t s); \
  void launch_p2_layout(bool to_device, const double* src, double* dst, int ne, int var,         \
                        const int* map, cudaStream_t s);                                         \
  size_t p2_tile_smem(int max_halo, int max_tasks);                                              \
  }
DGSWEM_DECLARE_P2_LAUNCHERS(fast_p2)
DGSWEM_DECLARE_P2_LAUNCHERS(strict_p2)
DGSWEM_DECLARE_P2_LAUNCHERS(mixed_p2)

// ---- discrete adjoint (adjoint.cu) ----------------------------------------
// Vector-Jacobian product of one RK stage's right-hand side L(q; n, HB) at
// stage state q: lam += (dL/dq)^T nu, g_n += (dL/dnbar)^T nu (element-mean
// Manning n), g_hb += (dL/dHB)^T nu.  Two kernels: per (edge, point) into
// the per-element scratch eb (each slot written by one thread), then per
// element (volume terms and the gather of eb).
struct AdjArgs {
  MeshView m;
  Physics ph;
  const double* __restrict__ q;         // stage state at which L was evaluated
  const double* __restrict__ nu;        // cotangent of L, 9*NE
  double* lam;                          // += (dL/dq)^T nu, 9*NE
  double* g_n;                          // += per element, or null (no Manning n)
  double* g_hb;                         // += [k*NE + e]
  const double* __restrict__ ocean_zg;  // this stage's ocean forcing (as StageArgs)
  const double* __restrict__ pr;        // nodal pressure (NWS=1), or null
  double rampdg;
  double* eb;                           // 36*NE scratch: edge-point trace cotangents
  const int* __restrict__ edges;        // (element, local edge) pairs: interior edges from the in side, boundary edges
  int nedge;
  const int* __restrict__ wd;           // WDFLG the stage kernel read (dry elements: no volume terms, dry-side edge rules)
};
// One stage of the reverse SSP-RK accumulation: lam_I += a_I lam_j and
// nu_I += b_I lam_j for I < n (b_I already times DT).
struct SspAdjArgs {
  const double* lam_j;
  double* lam[kMaxStages];
  double* nu[kMaxStages];
  double a[kMaxStages], b[kMaxStages];
  int n;
  int first;  // the step's first pass (j = NRK+1): assign instead of add (no zeroing beforehand)
  long long len;
};
namespace adj {
void set_basis(const BasisP1& b);
void launch_rhs_vjp(const AdjArgs& a, cudaStream_t s);
void launch_ssp_adj(const SspAdjArgs& a, cudaStream_t s);
// Reverse mode of the stage's SLOPELIMITER5 (slopeflag) and WETDRY (wetdry)
// with frozen branches at pre-limiter state qpre and input flags wd: lam
// (9*NE, in place) from the cotangent of the limited / wet-dried state to
// the pre-limiter state's; g_hb += the HB terms of WETDRY's flattening.
// Scratch: mm (6*NP), arg (6*NP), lb (18*NE), nb (6*NP).
void launch_limit_vjp(const MeshView& m, const Physics& ph, int slopeflag, int wetdry, const int* wd,
                      const double* qpre, double* mm, int* arg, double* lam, double* lb, double* nb, double* g_hb,
                      cudaStream_t s);
// eta[slot*ng + g] = sum_k phi[g*3+k] * q[k*NE + elem[g]] (ZE at gauge points)
void launch_gauge_eval(const double* q, int ne, const int* elem, const double* phi, int ng, double* eta,
                       cudaStream_t s);
// lam[k*NE + elem[g]] += phi[g*3+k] * w[g] (misfit seed of the ZE modes),
// over the gauge groups (distinct elements gel, CSR gptr / ggauge)
void launch_gauge_seed(double* lam, int ne, const int* gel, const int* gptr, const int* ggauge, const double* phi,
                       const double* w, int ngroup, cudaStream_t s);
}  // namespace adj

constexpr int kPointBlock = 256;

}  // namespace dgswem
