/*
 * dgswem_cuda.h -- C-ABI of the B200 DG hydro time step (drop-in boundary).
 *
 * The Fortran host replaces `CALL DG_HYDRO_TIMESTEP(IT)` (reference
 * src/DG_timestep.F:30) by `dgswem_cuda_hydro_timestep(h, IT)` through an
 * iso_c_binding interface, in the style of the reference's own C binding
 * (src/c_interface.F90:1-23, src/count_edges.cpp:324-354): plain pointers and
 * sizes, `int` scalars by value, no C++ or torch types.
 *
 * Array conventions follow the reference's Fortran declarations so a host
 * passes its module arrays unchanged (c_loc of the first element):
 *   - column-major, 1-based ids (node, element and edge numbers start at 1);
 *   - NM(NE,3)        -> nm[e + ne*v]
 *   - NEDNO(2,NEDGES) -> nedno[s + 2*ed]   (NEDEL, NEDSD likewise)
 *   - NELED(3,NE)     -> neled[l + 3*e]
 *   - ZE(DOFH,NE)     -> ze[k + dofh*e]    (one RK stage slice; QX, QY, HB)
 *   - EMO_DG(NBFR,NEEDS,2) -> emo_dg[f + nbfr*(l + needs*ipt)]
 * All reals are REAL(SZ) with SZ=8 (double).  Every entry point returns 0 on
 * success and a nonzero status otherwise; the library never aborts the
 * process; dgswem_cuda_last_error() gives the message.  There is no CPU
 * fallback: without a usable GPU, dgswem_cuda_create() fails.
 */
#ifndef DGSWEM_CUDA_H
#define DGSWEM_CUDA_H

#ifdef __cplusplus
extern "C" {
#endif

#define DGSWEM_CUDA_ABI_VERSION 1

enum {
  DGSWEM_OK = 0,
  DGSWEM_ERR_ARG = 1,      /* invalid argument or unsupported configuration */
  DGSWEM_ERR_CUDA = 2,     /* CUDA runtime error */
  DGSWEM_ERR_IO = 3,       /* input deck could not be read */
  DGSWEM_ERR_NUMERIC = 4   /* NaN / negative depth detected on the device */
};

/*
 * Setup data: what PREP_DG (reference src/prep_DG.F:25-1539) leaves in the
 * GLOBAL/DG/NodalAttributes modules, restricted to what the hydro step reads.
 * Pointers are only read during dgswem_cuda_create(); they are not retained.
 */
typedef struct dgswem_cuda_setup {
  /* sizes */
  int ne, np;              /* elements, nodes                              */
  int dofh;                /* modes per variable: 3 (p=1) or 6 (p=2)       */
  int nrk;                 /* RK stages (RK_STAGE)                         */
  int nedges;              /* NEDGES                                       */
  int nieds, nleds, needs, nfeds, nreds, nebseg, nibseg;
  /* switches (read_input.F, dgswem.F:131-170, fort.dg) */
  int ics;                 /* 1 Cartesian, 2 spherical (CPP)               */
  int nolifa;              /* >=2 enables WETDRY                           */
  int iflinbf, ifhybf;     /* friction form flags                          */
  int ifnlfa;              /* finite amplitude flag                        */
  int nramp;               /* ramp option                                  */
  int nws;                 /* 0 or 1 (met forcing via dgswem_cuda_set_met) */
  int rainfall;            /* 0 or 1                                       */
  int slopeflag;           /* 0 off, otherwise SLOPELIMITER5               */
  int load_manning;        /* ManningsN from fort.13                       */
  double nleq, leq;        /* nonlinear / linear switches                  */
  double g, h0, dtdp, statim, dramp;
  double cf, hbreak, ftheta, fgamma;
  double sfea0;            /* radians (ics=2)                              */
  /* SSP-RK coefficients (RK_TIME, prep_DG.F:1551-1990), row-major nrk*nrk:
   * atvd[(irk-1)*nrk + (i-1)] = ATVD(IRK,I); dtvd[irk-1] = DTVD(IRK)      */
  const double *atvd, *btvd, *dtvd;
  /* mesh */
  const int* nm;           /* NM(NE,3)                                     */
  const double *x, *y;     /* nodal coordinates (CPP metres if ics=2)      */
  const double* dp;        /* nodal depth after the H0 clamp               */
  /* edge graph (create_edge_data.F) */
  const int *nedno, *nedel, *nedsd, *neled;
  const int *niedn, *nledn, *needn, *nfedn, *nredn, *nebsegn;
  const int* nibsegn;      /* NIBSEGN(2,NIBSEG)                            */
  /* element data */
  const double* hb;        /* HB(DOFH,NE) bathymetry modes                 */
  const double* cori_el;   /* CORI_EL(NE)                                  */
  const double* fric_el;   /* FRIC_EL(NE)                                  */
  const double* manning;   /* ManningsN(NP) or NULL                        */
  /* initial state (stage 1 slice) */
  const double *ze, *qx, *qy;
  const int* wdflg;
  /* open-ocean harmonic forcing (prep_DG.F:180-205) */
  int nbfr;
  const double *amig, *ff, *face, *per;
  const double *emo_dg, *efa_dg;
  /* flow boundaries (prep_DG.F:208-245) */
  int nffr;
  const double *famig, *fff, *fface, *fper;
  const double *qnam_dg, *qnph_dg;   /* QNAM_DG(NFFR,NFEDS,2)              */
  /* barriers (read_input.F:2668-2685) */
  const double *ebht, *ebcfsp;       /* per external-barrier segment       */
  const double *ibht, *ibcfsb, *ibcfsp; /* per internal-barrier segment    */
} dgswem_cuda_setup;

typedef struct dgswem_cuda dgswem_cuda;

/* dgswem_cuda_create flags.  Default (0): the strict kernels, compiled with
 * -fmad=false so that every product and sum is rounded separately in the
 * reference's evaluation order, with the Manning depth factor
 * DEPTH**(1.D0/3.D0) correctly rounded: bit-identical to a non-contracting
 * FP64 CPU build of the reference path with correctly rounded pow (only the
 * hybrid friction's general pow may differ in the last bit).
 * DGSWEM_CUDA_STRICT names the default explicitly. */
#define DGSWEM_CUDA_STRICT 1
/* DGSWEM_CUDA_FAST: the same kernels compiled with fused multiply-add
 * contraction and cbrt for the Manning factor.  About 9 % faster per step;
 * results differ from the strict form by rounding, and the slope limiter's
 * and WETDRY's branch decisions amplify that difference at their ties
 * (1e-9..1e-5 relative after 10 steps of a wet/dry beach).  Excludes the
 * other flags. */
#define DGSWEM_CUDA_FAST 4
/* DGSWEM_CUDA_MIXED: mixed precision.  The stage kernel's edge traces,
 * numerical fluxes, boundary ghost states, volume fluxes and sources, the
 * right-hand-side sums and the slope limiter's clamp and redistribution
 * sweeps (on deviations from the element mean) run in FP32; the state
 * (ZE/QX/QY modes), the SSP-RK combination (so the element-mean elevation
 * accumulates across stages in FP64), the ocean depth-positivity fix, the
 * node min/max and WETDRY stay FP64; on a p=2 handle the right-hand-side
 * sums and their weights stay FP64 too (the hydrostatic pressure's edge and
 * volume integrals cancel to FP32 precision only with FP64 weights).
 * Results differ from the FP64 forms by the FP32 rounding.  Excludes the
 * other flags. */
#define DGSWEM_CUDA_MIXED 2

/* Copies the setup to GPU `device` and builds the device layout.
 * Replaces the state the reference keeps in module arrays after PREP_DG
 * (src/dgswem.F:196).  DOFH = 6 makes a p=2 handle (strict, fast or mixed):
 * no slope limiter and no wetting/drying (p=1 only in the reference), land,
 * ocean and interior edges, ICS=1, a whole-mesh handle; its interior-edge
 * sums run over all six modes (the reference's p=2 sums modes 1-3 only).
 * State arrays are ZE/QX/QY(6, NE).  The adjoint, state slots, tile shapes
 * and partitions are p=1 only and return DGSWEM_ERR_ARG on a p=2 handle.
 * A p=2 stage runs one tile kernel (edge fluxes kept in shared memory), or,
 * where a tile does not fit the device's shared memory or the environment
 * variable DGSWEM_CUDA_P2_PAIR is set to a non-zero integer at create, an
 * edge kernel and an element kernel with the edge-point fluxes in device
 * memory; the strict build gives the same bits with either.
 * The integer mesh tables are range-checked on the host before the device
 * is touched (NM in 1..NP, NELED and the boundary lists in 1..NEDGES, NEDEL
 * in 0..NE, NEDSD in 1..3 where NEDEL names an element): an inconsistent
 * mesh returns DGSWEM_ERR_ARG. */
int dgswem_cuda_create(const dgswem_cuda_setup* setup, int device, int flags,
                       dgswem_cuda** out);

/* ---- partitioned mesh (one handle per GPU) --------------------------------
 * The reference runs one MPI rank per METIS subdomain and exchanges ghost
 * elements after the SSP update and after the limiter/WETDRY
 * (DG_hydro_timestep.F:493-514, 555-579; messenger_elem.F).  Here partition
 * `part` of `nparts` owns a contiguous range of the elements' Morton order
 * and keeps ghost copies of its neighbours; the caller moves the halo
 * between handles (NCCL, peer copies, or device copies on one GPU) between
 * the stage calls:
 *
 *   for each RK stage irk:  stage_rhs(it, irk) on every partition
 *                           halo kind 0 (pack -> move -> unpack), if SLOPEFLAG
 *                           stage_limit(irk) on every partition
 *                           halo kind 1
 *   step_end() on every partition
 *
 * Halo kind 0: element means of ZE, QX, QY (3 doubles per element) of the
 * elements sharing a node with another partition's elements, read by that
 * partition's limiter node pass.  Kind 1: the nine modal values and WDFLG (10
 * doubles) of the elements sharing an edge (or an internal barrier) with
 * another partition's elements.  Buffers are device memory of the handle's
 * device; pack/unpack run on the handle's stream (dgswem_cuda_set_stream).
 * The state upload takes the whole input-order arrays (NE elements); the
 * download writes the owned elements' entries only.  dgswem_cuda_hydro_timestep,
 * dgswem_cuda_run and modal2nodal need a whole-mesh handle (nparts = 1).
 * No counterpart in the reference's C interface. */
int dgswem_cuda_create_part(const dgswem_cuda_setup* setup, int part, int nparts, int device,
                            int flags, dgswem_cuda** out);
int dgswem_cuda_part_info(const dgswem_cuda* h, int* part, int* nparts, int* n_owned,
                          int* n_local);
/* One RK stage's right-hand side and SSP update of the owned elements
 * (stage buffer irk, 1..NRK), then the limiter and WETDRY of the same stage,
 * then the end of the step (the stage-NRK+1 state becomes the step state). */
int dgswem_cuda_stage_rhs(dgswem_cuda* h, int it, int irk);
/* dgswem_cuda_stage_rhs in two launches, so that a partition's stage can
 * start while the halo exchange that refreshes its ghosts is in flight
 * (the overlap of the reference's persistent MPI requests,
 * src/messenger_elem.F:832-980): tiles = 1 runs the stage kernel on the tiles
 * that read no ghost element and no internal-barrier side (valid as soon as
 * the previous stage's limiter has run on this partition), tiles = 2 on the
 * others (after the ghosts are unpacked); tiles = 0 runs all, the same as
 * dgswem_cuda_stage_rhs.  A stage is either one call with 0 or a call with 1
 * followed by one with 2; results are bit-identical either way.
 * dgswem_cuda_tile_split gives the two tile counts.  No counterpart in the
 * reference's C interface. */
int dgswem_cuda_stage_rhs_tiles(dgswem_cuda* h, int it, int irk, int tiles);
int dgswem_cuda_tile_split(const dgswem_cuda* h, int* n_interior, int* n_boundary);
int dgswem_cuda_stage_limit(dgswem_cuda* h, int irk);
int dgswem_cuda_step_end(dgswem_cuda* h);
/* Elements this partition sends to / receives from `peer` for halo `kind`;
 * a buffer holds 3 (kind 0) or 10 (kind 1) doubles per element, in the order
 * of the peer's matching list (ascending input element ids). */
int dgswem_cuda_halo_count(const dgswem_cuda* h, int kind, int peer, int* nsend, int* nrecv);
int dgswem_cuda_halo_pack(dgswem_cuda* h, int kind, int peer, int irk, double* buf);
int dgswem_cuda_halo_unpack(dgswem_cuda* h, int kind, int peer, int irk, const double* buf);
/* Host-only: the input element ids (0-based, ascending) partition `part`
 * sends to / receives from `peer` for halo `kind` (NULL id arrays: counts
 * only).  Needs no GPU. */
int dgswem_part_halo_ids(const dgswem_cuda_setup* setup, int part, int nparts, int peer, int kind,
                         int* send_ids, int* nsend, int* recv_ids, int* nrecv);
void dgswem_cuda_destroy(dgswem_cuda* h);

/* One DG_HYDRO_TIMESTEP(IT) (src/DG_hydro_timestep.F:24-744): all RK stages,
 * slope limiter, wet/dry, stage copy.  Asynchronous on the library stream. */
int dgswem_cuda_hydro_timestep(dgswem_cuda* h, int it);
/* Steps it0 .. it0+nsteps-1 (one call per host loop, fewer launches). */
int dgswem_cuda_run(dgswem_cuda* h, int it0, int nsteps);
/* Waits for queued steps and reports device-side numeric errors. */
int dgswem_cuda_synchronize(dgswem_cuda* h);

/* Stage-1 state ZE/QX/QY(DOFH,NE) and WDFLG(NE), host memory.  Download is
 * the sync point, like `!$acc wait` at src/DG_timestep.F:32. */
int dgswem_cuda_upload_state(dgswem_cuda* h, const double* ze, const double* qx,
                             const double* qy, const int* wdflg);
int dgswem_cuda_download_state(dgswem_cuda* h, double* ze, double* qx, double* qy,
                               int* wdflg);

/* NWS=1: nodal WSX2/WSY2/PR2 (src/met_forcing.F:49-66); applied every stage
 * times RAMPDG.  Arrays of NP doubles. */
int dgswem_cuda_set_met(dgswem_cuda* h, const double* wsx2, const double* wsy2,
                        const double* pr2);

/* NWS = 1 from a fort.22 file, as MET_FORCING reads it (src/met_forcing.F:
 * 49-66): before every RK stage (src/DG_hydro_timestep.F:104) the handle
 * reads the next NP records "NHG, WSX2, WSY2, PR2" (list-directed, input node
 * order) and uploads them; the stage kernel applies the stage's RAMPDG, the
 * reference's RampMete.  From then on these fields replace those of
 * dgswem_cuda_set_met; a NULL path detaches the file (the last fields stay).
 * DGSWEM_ERR_IO when the file cannot be opened, ends inside a block or holds
 * a value that is not a number (the step that needed it reports it).  While a
 * file is attached, dgswem_cuda_run does not use CUDA graphs (the host reads
 * between stages) and the discrete adjoint is not available.  A partition
 * handle reads the whole mesh's NP records and keeps its own nodes'. */
int dgswem_cuda_met_file(dgswem_cuda* h, const char* path);

/* Host reader of the same records (no device): dgswem_met_reader_next fills
 * the next MET_FORCING block, NP values of each field in input node order;
 * dgswem_met_reader_calls counts the blocks read. */
typedef struct dgswem_met_reader dgswem_met_reader;
int dgswem_met_reader_open(const char* path, int np, dgswem_met_reader** out);
int dgswem_met_reader_next(dgswem_met_reader* r, double* wsx2, double* wsy2, double* pr2);
long dgswem_met_reader_calls(const dgswem_met_reader* r);
void dgswem_met_reader_close(dgswem_met_reader* r);

/* modal2nodal (src/write_results.F:14-170) on the device; results copied to
 * host arrays of NP entries (any may be NULL).  nodecode: 1 where a wet
 * element touches the node (the value WETDRY leaves in NODECODE). */
int dgswem_cuda_modal2nodal(dgswem_cuda* h, double* eta2, double* uu2, double* vv2,
                            int* nodecode);

/* Largest NP that dgswem_cuda_modal2nodal_noalloc accepts: its static device
 * scratch holds ETA2, UU2 and VV2 for this many nodes (24 MiB).  The CUDA
 * loader reserves those 24 MiB on every device where the library's device
 * code is loaded, whether or not dgswem_cuda_modal2nodal_noalloc is ever
 * called (every rank of a partitioned run holds them too). */
#define DGSWEM_CUDA_NOALLOC_MAX_NODES (1 << 20)

/* dgswem_cuda_modal2nodal that allocates nothing, for p=1 whole-mesh handles
 * (a p=2 or a partition handle: DGSWEM_ERR_ARG).  No counterpart in the
 * reference (its modal2nodal fills the host arrays directly).  Same kernel and
 * same results as dgswem_cuda_modal2nodal, but the nodal scratch is a static
 * device array of DGSWEM_CUDA_NOALLOC_MAX_NODES nodes instead of the handle's
 * staging buffer, which dgswem_cuda_modal2nodal grows (cudaFree + cudaMalloc)
 * when 4 NP exceeds it.  For hosts that must not allocate or free device
 * memory once the time loop runs: a host sharing the GPU with work on its own
 * streams (cudaFree waits for the whole device) or one that has reserved the
 * rest of HBM for its own pool (the allocation could fail mid-run).
 * - NP > DGSWEM_CUDA_NOALLOC_MAX_NODES: DGSWEM_ERR_ARG, nothing launched.
 * - The first call on each device looks up the scratch's device address
 *   (cudaGetSymbolAddress, which may load the library's device module); make
 *   that first call before any stream capture.  The address is kept for the
 *   life of the process: it assumes the device's primary context is not
 *   destroyed and recreated (cudaDeviceReset) between calls.
 * - Any of the four outputs may be NULL (that copy is skipped).
 * - Nothing in the scratch has to start at zero: the kernel writes all NP
 *   entries of each nodal array before they are copied out.
 * - All handles on one device share the one scratch array: calls that overlap
 *   in time on the same device (from several host threads) race on it and
 *   must be serialised by the caller. */
int dgswem_cuda_modal2nodal_noalloc(dgswem_cuda* h, double* eta2, double* uu2, double* vv2,
                                    int* nodecode);

/* Number of kernels the library launched since create (for accounting). */
long long dgswem_cuda_kernel_launches(const dgswem_cuda* h);

/* Run the whole-step chunks of dgswem_cuda_run as CUDA graphs of `steps`
 * steps (even, >= 2; 0: off, the default): the chunk's stage kernels and one
 * copy of its host forcing and ramps are captured once, then replayed, so a
 * chunk costs one graph launch instead of 3 x NRK kernel launches per step.
 * Results are bit-identical to the launches without graphs.  Not while
 * per-kernel profiling is on.  No counterpart in the reference. */
int dgswem_cuda_set_graph(dgswem_cuda* h, int steps);

/* ---- tile and block shapes, autotuner ------------------------------------
 * The stage kernel is compiled for several tile shapes (elements per tile,
 * threads per block) and the limiter / WETDRY kernel for several block
 * sizes; every shape gives bit-identical results.  dgswem_cuda_shapes lists
 * them (arrays of up to DGSWEM_CUDA_MAX_SHAPES entries, any may be NULL;
 * a limiter shape is its threads per block and the resident blocks per SM
 * its registers were allocated for).
 * dgswem_cuda_set_shapes selects one of each by index (-1 keeps the current
 * one) and rebuilds the stage tile plan; DGSWEM_ERR_ARG if the tile shape's
 * plan does not fit the mesh (the current plan stays).  Captured CUDA graphs
 * are released.  dgswem_cuda_get_shapes reports the current indices; for a
 * p=2 handle the tile shape is that of the p=2 tile kernel's plan, or -1
 * when the mesh's tiles do not fit shared memory and the p=2 edge + element
 * kernel pair runs instead.
 *
 * dgswem_cuda_autotune times `steps` whole steps from step `it` (forcing of
 * steps it..it+steps-1), best of `reps`, with each tile shape, then with
 * each limiter block size under the fastest tile shape, every timing from
 * the handle's current state; it restores that state (ZE, QX, QY, WDFLG and
 * the NaN flag) and keeps the fastest shapes.  ms_tile / ms_limit (NULL or
 * arrays of the shape counts) receive milliseconds per step, -1 for a shape
 * not timed (its plan does not fit, or no limiter / WETDRY runs).  With
 * DGSWEM_CUDA_TUNE_CACHED a result measured earlier in this process for the
 * same mesh signature (variant, device, sizes, edge graph, physics
 * switches) is reused without timing.  Whole-mesh handles only
 * (dgswem_cuda_create).  No counterpart in the reference. */
#define DGSWEM_CUDA_MAX_SHAPES 8
#define DGSWEM_CUDA_TUNE_CACHED 1
int dgswem_cuda_shapes(int* n_tile, int* tile_elems, int* tile_threads, int* n_limit, int* limit_threads,
                       int* limit_blocks_per_sm);
int dgswem_cuda_set_shapes(dgswem_cuda* h, int tile_shape, int limit_shape);
int dgswem_cuda_get_shapes(const dgswem_cuda* h, int* tile_shape, int* limit_shape);
int dgswem_cuda_autotune(dgswem_cuda* h, int it, int steps, int reps, int flags, double* ms_tile,
                         double* ms_limit);

/* Launch on the caller's CUDA stream (a cudaStream_t passed as void*, used
 * as given: NULL is the CUDA default stream).  dgswem_cuda_stream() returns
 * the stream in use, so a caller can restore the library's own stream.
 * Lets a host time the step with its own events or order it after its own
 * work.  No counterpart in the reference (its OpenACC regions run on async
 * queue 1). */
int dgswem_cuda_set_stream(dgswem_cuda* h, void* stream);
void* dgswem_cuda_stream(const dgswem_cuda* h);

/* Per-kernel timing with CUDA events recorded around every launch on the
 * launching stream.  enable != 0 starts accumulating (and resets); read
 * returns, per kernel kind (0 stage, 1 node_minmax, 2 limit_wetdry,
 * 3 other), the summed milliseconds and launch counts (arrays of 4). */
int dgswem_cuda_profile(dgswem_cuda* h, int enable);
int dgswem_cuda_profile_read(dgswem_cuda* h, double* ms, long long* launches);

/* Last error message of the calling thread (NUL-terminated, truncated). */
int dgswem_cuda_last_error(char* buf, int buflen);

/* ---- parameters, state slots, gauges, discrete adjoint ---------------------
 * No counterparts in the reference.  All need a whole-mesh handle
 * (dgswem_cuda_create).
 *
 * dgswem_cuda_set_params: replace the element-mean Manning n (nbar[NE], input
 * element order; the deck must have nodal Manning n) and/or the bathymetry
 * modes (hb = HB(DOFH,NE)); NULL keeps a field.  WETDRY keeps reading the
 * nodal depths DP of the setup.
 *
 * dgswem_cuda_state_save / _load: copy the current state (ZE/QX/QY, WDFLG)
 * to / from device slot `slot` (allocated on first save; checkpoints).
 *
 * dgswem_cuda_gauges: ng gauge points, each in element elem[g] (1-based
 * input id) with ZE basis values phi[3g..3g+2] at the point (1 and the
 * corner-map combinations of its barycentric weights); dgswem_cuda_gauge_eta
 * evaluates ZE of the current state there.
 *
 * Discrete adjoint of DG_HYDRO_TIMESTEP (NLEQ=1, ICS=1, land and ocean
 * edges, slope limiter 5 and WETDRY with their branches frozen at the
 * forward's, linear / quadratic / Manning friction; DGSWEM_ERR_ARG otherwise;
 * FP64 handles only):
 *   dgswem_cuda_adjoint_begin   zero the state cotangent and the gradients
 *   dgswem_cuda_adjoint_seed    add w[g] * dZE(gauge g)/dq to the cotangent of
 *                               the state the next adjoint step ends at
 *   dgswem_cuda_adjoint_step    with the state before step `it` loaded,
 *                               recompute step `it` (the handle ends at the
 *                               state after it) and carry the cotangent back
 *                               through it, adding that step's parameter
 *                               gradient
 *   dgswem_cuda_adjoint_read    gradients w.r.t. nbar (NE, input order) and HB
 *                               (HB(DOFH,NE)), and the current state
 *                               cotangent (ZE/QX/QY(DOFH,NE)); NULL skips. */
int dgswem_cuda_set_params(dgswem_cuda* h, const double* nbar, const double* hb);
int dgswem_cuda_state_save(dgswem_cuda* h, int slot);
int dgswem_cuda_state_load(dgswem_cuda* h, int slot);
int dgswem_cuda_gauges(dgswem_cuda* h, int ng, const int* elem, const double* phi);
int dgswem_cuda_gauge_eta(dgswem_cuda* h, double* eta);
int dgswem_cuda_adjoint_begin(dgswem_cuda* h);
int dgswem_cuda_adjoint_seed(dgswem_cuda* h, const double* w);
int dgswem_cuda_adjoint_step(dgswem_cuda* h, int it);
int dgswem_cuda_adjoint_read(dgswem_cuda* h, double* g_nbar, double* g_hb, double* lam_ze, double* lam_qx,
                             double* lam_qy);
/* The two passes of a gauge-misfit gradient with sqrt(N)-style checkpoints,
 * each one call.  dgswem_cuda_misfit_forward runs steps it0 .. it0+nsteps-1
 * from the current state, saving the state every `every` steps in slots
 * 0, 1, .. and writing ZE at the gauges after each step to eta[k*ng + g].
 * dgswem_cuda_adjoint_sweep (after it, same it0 / nsteps / every) zeroes the
 * gradients and carries w[k*ng + g] (the misfit's derivative with respect to
 * ZE at gauge g after step k) back to the initial state: per segment it
 * re-runs the steps from the checkpoint keeping their stage states (slots
 * from nseg on, and `every` x (NRK-1) stage buffers), then steps back.
 * Read the result with dgswem_cuda_adjoint_read. */
int dgswem_cuda_misfit_forward(dgswem_cuda* h, int it0, int nsteps, int every, double* eta);
/* Building blocks of the reverse mode.  dgswem_cuda_limit_state applies the
 * stage path's SLOPELIMITER5 and WETDRY (those the deck turns on) to the
 * current state in place.  dgswem_cuda_limiter_vjp returns, at the current
 * state and WDFLG as their input, the transpose of the two with their
 * branches frozen applied to the cotangents lam_* of their output
 * (ZE/QX/QY(DOFH,NE) in, the same layout out); needs SLOPEFLAG != 0 or
 * WETDRY, and the adjoint's scope. */
int dgswem_cuda_limit_state(dgswem_cuda* h);
int dgswem_cuda_limiter_vjp(dgswem_cuda* h, const double* lam_ze, const double* lam_qx, const double* lam_qy,
                            double* out_ze, double* out_qx, double* out_qy);
int dgswem_cuda_adjoint_sweep(dgswem_cuda* h, int it0, int nsteps, int every, const double* w);

/* ---- standalone input path (no Fortran host) ------------------------------
 * Reads fort.14, fort.15, fort.dg (and fort.13 when NWP>0) from `dir` and runs
 * the setup the reference does in READ_INPUT + PREP_DG, producing a
 * dgswem_cuda_setup.  The deck owns all arrays the setup points to. */
typedef struct dgswem_deck dgswem_deck;
int dgswem_deck_open(const char* dir, dgswem_deck** out);
const dgswem_cuda_setup* dgswem_deck_setup(const dgswem_deck* d);
/* nt, nspoolge, ntcysge, ntcyfge, noutge (integer run controls) */
int dgswem_deck_int(const dgswem_deck* d, const char* key, int* value);
void dgswem_deck_close(dgswem_deck* d);

/* ---- ensembles (no counterpart in the reference: one mesh per run there) ---
 * Merges n setups into one deck whose setup holds the n meshes side by side:
 * element, node and edge arrays concatenated in member order, ids offset by
 * the preceding members' counts (member i's elements are ids
 * sum(ne[0..i-1]) + 1 ..).  A handle created from it advances every member
 * in each kernel launch.  Time step, RK tables, physics switches and
 * constants and the tidal / flow constituents must be equal across members
 * (DGSWEM_ERR_ARG otherwise); amplitudes per boundary edge, Manning n per
 * node and met fields per node may differ.  The merged deck owns copies;
 * the members may be closed afterwards.  Run controls (dgswem_deck_int) of
 * the merged deck are 0. */
int dgswem_deck_merge(const dgswem_cuda_setup* const* parts, int n, dgswem_deck** out);

#ifdef __cplusplus
}
#endif
#endif /* DGSWEM_CUDA_H */
