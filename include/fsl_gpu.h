/*
 * fsl_gpu.h -- C ABI of the B200 (sm_100a) explicit time step of the
 * freeShearLayer compressible LES solver.
 *
 * The reference's "operator API" for this path is the set of global void
 * functions its ANSI-C driver calls once per stage (src/layer2.c:141-185),
 * all communicating through globals (src/global.h:6-72).  This header gives
 * the same entry points with explicit state: one fsl_ctx owns one
 * device-resident domain (the five conserved variables, the stage buffer, the
 * SGS viscosity and the boundary data) on the current CUDA device, and every
 * call works on that context's single CUDA stream.
 *
 * Conventions (all entry points):
 *   - return FSL_OK (0) on success or a negative FSL_ERR_* code; no call
 *     exits the process (the reference calls exit(-1), src/helpers.c:63-76);
 *   - calls on one context are not thread-safe; contexts are independent;
 *   - the product has no CPU fallback: without a usable sm_100 device
 *     fsl_init returns FSL_ERR_NODEVICE;
 *   - host arrays are plain C arrays of double; no pointer is retained.
 *
 * Layouts:
 *   state   : the interior in the reference's backup.dat row layout
 *             (src/finalize.c:22-29): for i in 1..LEN, for j in 1..HIG:
 *             DEP values of rho, then rho u, rho v, rho w, E.
 *   padded  : (LEN+2)(HIG+2)(DEP+2) doubles, k fastest -- the reference's
 *             Array3D(LEN+2,HIG+2,DEP+2) (src/helpers.c:58-80) flattened.
 *   faces   : dense over the reference's face index ranges,
 *             x (LEN+1)*HIG*DEP, y LEN*(HIG+1)*DEP, z LEN*HIG*(DEP+1).
 */
#ifndef FSL_GPU_H
#define FSL_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define FSL_ABI_VERSION 1

/* return codes */
#define FSL_OK 0
#define FSL_ERR_ARG (-1)         /* invalid argument or parameter set */
#define FSL_ERR_NOMEM (-2)       /* device or host allocation failed */
#define FSL_ERR_CUDA (-3)        /* a CUDA runtime call failed */
#define FSL_ERR_NONFINITE (-4)   /* non-finite state, non-positive density or Courant max */
#define FSL_ERR_TIMEOUT (-5)     /* a bounded device wait gave up */
#define FSL_ERR_IO (-6)          /* file could not be opened or parsed */
#define FSL_ERR_UNSUPPORTED (-7) /* option combination not available */
#define FSL_ERR_NODEVICE (-8)    /* no usable sm_100 CUDA device */

/* boundary setups */
#define FSL_SETUP_SPATIAL 0  /* the reference's BCs: step inflow / outflow in x, slip y, periodic z */
#define FSL_SETUP_TEMPORAL 1 /* temporal shear layer: periodic x and z, zero-gradient y */

/* Courant-number definitions */
#define FSL_CFL_STREAMWISE 0 /* max of u dt/dx (src/helpers.c:31-43) */
#define FSL_CFL_ACOUSTIC 1   /* max of dt((|u|+c)/dx + (|v|+c)/dy + (|w|+c)/dz) */

/* arithmetic of the stage update */
#define FSL_PREC_FP64 0 /* plain method: FP64 throughout, reference evaluation order */
#define FSL_PREC_FP32 1 /* FP32 bulk, FP64 U^n, RK combination, dt reduction and sums */

/* subgrid closure */
#define FSL_SGS_DYNAMIC 0 /* dynamic Smagorinsky (Germano-Lilly), src/turbulence.c:103-507 */
#define FSL_SGS_LEARNED 1 /* per-cell MLP Cs^2 with the dynamic procedure as judge */
#define FSL_SGS_STATIC 2  /* static Smagorinsky, rho_face Cs DD |S|_face per face: the reference's
                             DynamicSmagorinskySGS 0 branch (src/fluxes.c:193-205, :362-374,
                             :533-545), live in src-par (src-par/def.h:47); Cs from layer2.ini */
#define FSL_SGS_NONE 3    /* no SGS viscosity (mu_SGS = 0) */

/* reconstruction */
#define FSL_RECON_CHARMINMOD 0 /* characteristic kappa=1/3 minmod(beta=4), src/reconstruction.c:26-345 */
#define FSL_RECON_PPM 1        /* Colella-Woodward PPM on the same characteristic variables (project
                                  extension): the fused step in FP64 and FP32 bulk, and the per-phase
                                  FP64 kernels; cells next to a boundary keep the reference scheme */

/* Parameters: the 22 positional values of layer2.ini in file order
 * (src/initialize.c:25-58; src-par's mpi_layer2.bin holds the same 22 values
 * as float32), followed by the options that have no counterpart in the ini. */
typedef struct fsl_params {
    int LEN, HIG, DEP;
    double deltaX, deltaY, deltaZ, deltaT;
    int Answer, numstep;
    double mu_L, Pr_L, Pr_T, Cs;
    int BL_HIG;
    double Ua, Va, Wa;
    int Ns_min, Nst, f_step, nStages;
    double maxCoNum;
    /* options */
    int setup;       /* FSL_SETUP_* */
    int cfl_mode;    /* FSL_CFL_* */
    double seed_X;   /* disturbance RNG seed; the reference reads it from stdin (src/layer2.c:130) */
    int precision;   /* FSL_PREC_* */
    int sgs;         /* FSL_SGS_* */
    int recon;       /* FSL_RECON_* */
    int reserved[8];
} fsl_params;

typedef struct fsl_ctx fsl_ctx;

/* Scalars of the driver state, read with fsl_get_info. */
typedef struct fsl_info {
    double deltaT, deltaT_X, deltaT_Y, deltaT_Z; /* current time step and ratios */
    double maxCo;                                /* last Courant maximum */
    double X;                                    /* disturbance RNG state */
    double Ud, Vd, Wd;                           /* current disturbance velocities */
    unsigned k_min, k_max;                       /* current disturbance span */
    unsigned step;                               /* completed steps */
    int counter;                                 /* disturbance block countdown */
    int cur;                                     /* 0: U*_ = U, 1: U*_ = stage buffer */
    double DD, lambda_L, cp_Pr_T;                /* derived constants */
    unsigned long long device_bytes;             /* device memory held by the context */
} fsl_info;

/* ---- parameters ------------------------------------------------------- */

/* The reference's shipped layer2.ini physics with nStages = 3, FP64,
 * dynamic Smagorinsky, spatial setup, streamwise CFL. */
int fsl_params_default(fsl_params *p);
/* Parse layer2.ini: 22 positional lines read with atoi/atof, trailing text
 * ignored (replaces Initialize(), src/initialize.c:17-58).  Only the 22 ini
 * values of *p are written; its option fields are left as the caller set
 * them (initialise *p with fsl_params_default first). */
int fsl_params_from_ini(const char *path, fsl_params *p);
/* Parse mpi_layer2.bin: 22 float32 values in ini order
 * (src-par/initialize.c:35-81, written by src-par/ini2bin/ini2bin.c:63-64).
 * Option fields are left as for fsl_params_from_ini. */
int fsl_params_from_bin(const char *path, fsl_params *p);
/* Check a parameter set: FSL_OK or FSL_ERR_ARG. */
int fsl_params_check(const fsl_params *p);

/* ---- initial states (host arrays in the state layout) ----------------- */

/* The reference's fresh-start state, src/initialize.c:159-187. */
int fsl_initial_state(const fsl_params *p, double *state);
/* Temporal shear layer: u = dU/2 tanh(2y/delta_w0) about the domain centre,
 * p = 1e5 Pa, free-stream density 1 kg/m^3, Crocco-Busemann temperature,
 * dU = 2 Mc c_inf, uniform velocity perturbations of amplitude amp*dU from
 * splitmix64(seed).  *dU receives the velocity difference. */
int fsl_temporal_state(const fsl_params *p, double Mc, double delta_w0, double amp,
                       unsigned long long seed, double *state, double *dU);

/* ---- context ------------------------------------------------------------ */

/* Allocate a domain on the current CUDA device.  Replaces the allocation
 * part of Initialize() (src/initialize.c:97-125). */
int fsl_init(const fsl_params *p, fsl_ctx **ctx);
int fsl_destroy(fsl_ctx *ctx);
/* Message of the last error on this context (static storage, never NULL). */
const char *fsl_last_error(const fsl_ctx *ctx);
int fsl_get_info(fsl_ctx *ctx, fsl_info *info);
/* Block until the context's stream is idle.  FSL_ERR_NONFINITE when a
 * Courant reduction since the last fsl_upload_state met a density that is not
 * positive or a maximum that is not positive and finite (the flag is kept
 * until the next fsl_upload_state). */
int fsl_sync(fsl_ctx *ctx);

/* Upload/download U^n (backup.dat layout; src/initialize.c:134-148 reads,
 * src/finalize.c:22-29 writes). */
int fsl_upload_state(fsl_ctx *ctx, const double *state);
int fsl_download_state(fsl_ctx *ctx, double *state);
/* Set step counter and time step as a restart would (src/initialize.c:149-152). */
int fsl_set_time(fsl_ctx *ctx, unsigned step, double deltaT);
/* The same transfers without blocking the host, overlapped with the device
 * work around them: the upload's host-to-device copy and the download's
 * device-to-host copy run on copy streams of their own (one per direction,
 * with their own staging buffers), ordered against the context's stream by
 * events, so that a step's upload, the previous step's download and the step
 * itself proceed together.  `state` should be pinned host memory (pageable
 * memory works, without overlap) and must stay untouched until
 * fsl_transfer_wait returns. */
int fsl_upload_state_async(fsl_ctx *ctx, const double *state);
int fsl_download_state_async(fsl_ctx *ctx, double *state);
int fsl_transfer_wait(fsl_ctx *ctx);

/* ---- x-slabs (replaces src-par's MPI decomposition) ------------------------
 * A domain of LEN planes split along x into slabs, one context per slab (one
 * per GPU).  A slab context holds its owned planes plus W overlap planes on
 * each side (x-periodic temporal setup; in the spatial setup none before the
 * first slab and none after the last), in ascending global order, so that a
 * slab whose overlap wraps across the periodic seam has the seam on its own
 * periodic boundary, as the undivided domain does.  Once per step the overlap
 * planes are refreshed from the slabs that own them, and the Courant maximum
 * over the owned planes is combined across slabs by a maximum
 * (src-par/helpers.c:44, MPI_Allreduce MAX).  One step changes a plane only
 * through planes within 7 of it (9 with PPM; measured), so W >= 8
 * (10) keeps the owned planes bit-identical to the undivided domain.  This
 * takes the place of the per-stage ghost-plane messages of
 * src-par/boundCondInGhostCells.c:23-102, src-par/boundCondOnInterfaces.c:20-99
 * and src-par/communication.c:6-93.  Alternatively, as src-par does, the
 * overlap is refreshed after every stage (fsl_step_stage): one stage reaches
 * 3 planes (measured), so W >= 4.
 *
 * Planes are 1-based interior x-indices; buffers hold n planes in the
 * upload/download layout ([n][HIG][5][DEP] doubles), host or device memory
 * (copied with cudaMemcpyDefault; the call returns with the copy done).
 * Between steps they access U^n; while fsl_step_stage is in the middle of a
 * step, the current stage state (the output of stage 1 or 2), so that a slab
 * can refresh its overlap planes after every stage. */
int fsl_get_planes(fsl_ctx *ctx, int i0, int n, double *buf);
int fsl_set_planes(fsl_ctx *ctx, int i0, int n, const double *buf);
/* The same, queued on the context's stream without waiting (buf: device or
 * pinned host memory, untouched by the caller until the stream has reached
 * the copy).  Between contexts the caller orders the streams (fsl_stream and
 * CUDA events): a set after the get that filled its buffer, the next get into
 * a buffer after the set that read it. */
int fsl_get_planes_async(fsl_ctx *ctx, int i0, int n, double *buf);
int fsl_set_planes_async(fsl_ctx *ctx, int i0, int n, const double *buf);
/* Planes i0..i1 enter the Courant maximum (default 1..LEN).  A context with a
 * narrower range is an x-slab: fsl_step / fsl_step_phased then take one step
 * per call and, like the first fsl_step_stage of a step, need a combined
 * maximum (below) before each; a learned closure must have judgements off. */
int fsl_set_courant_range(fsl_ctx *ctx, int i0, int i1);
/* Make the owned Courant maximum of U^n available (a reduction, unless the
 * last step's final stage already accumulated it). */
int fsl_courant_prepare(fsl_ctx *ctx);
/* Read / replace that maximum (host round trip; replacing it with the
 * maximum over all slabs lets the next step rescale deltaT as one domain). */
int fsl_get_courant_max(fsl_ctx *ctx, double *maxCo);
int fsl_set_courant_max(fsl_ctx *ctx, double maxCo);
/* The same maximum in device memory as the bit pattern of the non-negative
 * double (unsigned 64-bit; such doubles order like their bit patterns), for
 * an in-place all-reduce MAX on the context's stream. */
unsigned long long *fsl_courant_bits(fsl_ctx *ctx);

/* ---- the driver's per-step scalar work ---------------------------------- */

/* checkCoNum(), src/helpers.c:23-52: reduce the Courant maximum over U^n on
 * the device, rescale deltaT to maxCoNum.  maxCo and dt may be NULL.
 * Returns FSL_ERR_NONFINITE when the maximum is not positive and finite. */
int fsl_check_courant(fsl_ctx *ctx, double *maxCo, double *dt);
/* The driver's disturbance-block draw, src/layer2.c:152-162 (host RNG,
 * src/helpers.c:13-17). */
int fsl_draw_disturbance(fsl_ctx *ctx);
/* Set the disturbance block directly (k span and velocities). */
int fsl_set_disturbance(fsl_ctx *ctx, unsigned k_min, unsigned k_max, double Ud, double Vd,
                        double Wd);

/* ---- per-phase entry points (reference names) ---------------------------
 * Each works on the current-stage buffer U*_ exactly like the reference
 * phase; they are the unfused path used for per-phase parity.  fsl_fluxes
 * does not recompute the SGS viscosity (the reference's Fluxes() calls
 * DynamicSmagorinsky first, src/fluxes.c:52-54); call
 * fsl_dynamic_smagorinsky first to reproduce Fluxes() exactly. */
int fsl_ghost_bc(fsl_ctx *ctx);            /* BounCondInGhostCells, src/boundCondInGhostCells.c:10 */
int fsl_reconstruct(fsl_ctx *ctx);         /* Reconstruction, src/reconstruction.c:26 */
int fsl_interface_bc(fsl_ctx *ctx);        /* BounCondOnInterfaces, src/bounCondOnInterfaces.c:11 */
int fsl_dynamic_smagorinsky(fsl_ctx *ctx); /* DynamicSmagorinsky(U1..U4,mu_SGS), src/turbulence.c:103 */
int fsl_fluxes(fsl_ctx *ctx);              /* Fluxes face loops, src/fluxes.c:57-571 */
int fsl_evolution(fsl_ctx *ctx, int stage); /* Evolution(nStages, Stage), src/evolution.c:15 */

/* SGS viscosity without any device allocation.  No counterpart in the
 * reference (which allocates 42 fresh arrays per call); it exists for callers
 * that cannot allocate device memory themselves or through this library: a
 * host application whose own allocator has reserved the device memory
 * up front, or a time-critical loop that must not stall on cudaFree's
 * device-wide synchronisation.
 *
 * Same arithmetic as fsl_dynamic_smagorinsky (bit-identical mu).  U: device
 * pointer to four consecutive (LEN+2)(HIG+2)(DEP+2) double arrays rho, rho u,
 * rho v, rho w (k fastest, ghost layer filled, e.g. by fsl_ghost_bc); mu:
 * device pointer to one such array, fully written (interior values, ghost
 * layer 0).  stream: a cudaStream_t of the current device (another device's
 * stream returns FSL_ERR_ARG), or NULL for the legacy default stream.  A CUDA
 * error left pending by earlier work returns FSL_ERR_CUDA before any work and
 * stays pending for its owner.
 *
 * Scratch is a fixed static device array of FSL_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until process exit; it needs
 * 40 (LEN+2)(HIG+2)(DEP+2) doubles, so (LEN+2)(HIG+2)(DEP+2) may be at most
 * FSL_NOALLOC_MAX_CELLS (e.g. 64x32x32 fits); larger sizes return
 * FSL_ERR_TOO_LARGE before any device work.  The call allocates nothing: no
 * cudaMalloc, no cudaFree, no library allocator.  The first call on a device
 * looks up the scratch address for that device (cudaGetSymbolAddress, with
 * that device current); make that first call before any stream capture.
 * All calls share the one scratch array, which keeps the previous call's
 * contents (the call clears what must start at zero): calls that overlap on
 * the GPU (different streams, or different host threads) race on it. */
#define FSL_ERR_TOO_LARGE (-9)
#define FSL_NOALLOC_SCRATCH_BYTES (32u << 20)
#define FSL_NOALLOC_MAX_CELLS (FSL_NOALLOC_SCRATCH_BYTES / (40u * 8u))
int fsl_dynamic_smagorinsky_noalloc(const double *U, double *mu, int LEN, int HIG, int DEP, double deltaX,
                                    double deltaY, double deltaZ, void *stream);

/* ---- whole steps ---------------------------------------------------------
 * nsteps iterations of the driver loop body without I/O (src/layer2.c:147-178):
 * Courant check and dt rescale, disturbance draw, nStages stages.  Uses the
 * fused stage kernels (nStages = 2 runs the per-phase kernels, FP64 only);
 * the SGS viscosity is evaluated once per step (it
 * depends only on U^n, src/fluxes.c:53, so this equals the reference's
 * per-stage evaluation).  Asynchronous: returns after queuing the work. */
int fsl_step(fsl_ctx *ctx, int nsteps);
/* Same work through the per-phase entry points (reference phase order). */
int fsl_step_phased(fsl_ctx *ctx, int nsteps);
/* One RK stage of fsl_step's work per call, the three stages in turn (nStages
 * = 3): the first call begins a step (Courant rescale, disturbance draw, SGS
 * viscosity, stage 1), the third completes it.  Same launches and results as
 * fsl_step.  Between the calls only fsl_get_planes / fsl_set_planes may touch
 * the state (the per-stage ghost-plane exchange of
 * src-par/boundCondInGhostCells.c:60-73); fsl_step, fsl_step_phased, the
 * Courant calls (fsl_check_courant, fsl_courant_prepare,
 * fsl_set_courant_max) and ensemble steps refuse with FSL_ERR_ARG until the
 * step is complete.  An upload abandons it (its deltaT rescale, step count
 * and disturbance draw stand, as after a completed step). */
int fsl_step_stage(fsl_ctx *ctx);

/* Launch-shape knobs of the fused kernels.  FP64 results do not depend on
 * them; FP32-bulk results may differ in the last bits (the compiler may
 * contract a flux into FMAs differently where a block's march starts). */
#define FSL_TUNE_STAGE_ROWS 1 /* rows per ring stage tile incl. 2 halo rows: 8, 12 or 16; or 0, the
                                 full-lane persistent 16 x 32 tile (the FP32 bulk's default with the
                                 reference reconstruction; elsewhere 0 runs 16) */
#define FSL_TUNE_STAGE_SEG 2  /* x planes marched per ring-tile stage block (default 48 FP32 bulk, 32 FP64;
                                 the full-lane tile splits the planes among its blocks itself) */
#define FSL_TUNE_CLOSURE_POLY 3 /* learned-closure inference: of every 8 SiLU value pairs, how many take
                                   the FMA-pipe polynomial tanh instead of the MUFU one: 0 or 2..6
                                   (default 2: 1.94 ms per step at 512x256x256 against 1.97 for 3;
                                   0, every pair on the MUFU pipe, runs about 10 % slower) */
int fsl_tune(fsl_ctx *ctx, int key, int value);

/* ---- debug bounds checks ---------------------------------------------------
 * libfsl_gpu_checked.so (`make -C freeshearlayer_b200 checked`) is this
 * library built with the global-memory indices of the step's kernels tested
 * against the extent of the array they index: the fused stage kernels (ring
 * tile and full lane, both precisions, ensembles), the per-phase kernels, the
 * dynamic procedure (both precisions), the closure's features and inference,
 * the Courant and conservation reductions, the state scatter/gather and the
 * probe and Tecplot kernels.  An offending access is counted, the first one of
 * each source file recorded, and the access redirected to element 0 of that
 * array, so it never leaves the allocation.  No counterpart in the reference
 * (its arrays are unchecked C). */
typedef struct fsl_bounds_report {
    unsigned long long hits; /* offending accesses since the last clear, all files */
    int unit;                /* file of the first one reported: 1 fsl_fused.cu, 2 fsl_fused32.cu,
                                3 fsl_mlp.cu, 4 fsl_phase.cu, 5 fsl_dyn32.cu, 6 fsl_io.cu;
                                0 when hits is 0 */
    int line;                /* its source line (in the file or a header it includes) */
    long long index, extent; /* the index and the extent it was checked against */
} fsl_bounds_report;
/* Synchronise the current device, then report (and with clear != 0 reset)
 * the records of every checked file; the first offending access reported is
 * that of the lowest-numbered file with one.  FSL_ERR_UNSUPPORTED in the
 * product build, which has no checks. */
int fsl_debug_bounds(fsl_bounds_report *out, int clear);

/* ---- debug / parity access ----------------------------------------------- */

/* which: 0 = U^n, 1 = stage buffer, 2 = current-stage buffer, 3 = mu_SGS. */
int fsl_get_cells(fsl_ctx *ctx, int which, int var, double *padded);
int fsl_set_cells(fsl_ctx *ctx, int which, int var, const double *padded);
/* dir 0/1/2; side 0 = minus-side state (flux after fsl_fluxes), 1 = plus-side. */
int fsl_get_faces(fsl_ctx *ctx, int dir, int side, int var, double *faces);
int fsl_set_faces(fsl_ctx *ctx, int dir, int side, int var, const double *faces);
/* Point U*_ at U^n (0) or at the stage buffer (1). */
int fsl_set_cur(fsl_ctx *ctx, int which);

/* ---- driver files ------------------------------------------------------------
 * real_bytes: 4 = the reference's shipped float `real` (src/type.h:4), 8 = FP64. */
/* backup.dat as Finalize() writes it (src/finalize.c:14-35): per (i, j) the DEP
 * values of U1..U5, then deltaT, then step (int).  fsl_read_backup restores
 * state, deltaT and step; src/initialize.c:133-158 skips deltaT and reads step
 * from its first bytes, which this reader does not copy.  FSL_ERR_IO when the
 * file size does not match the grid. */
int fsl_write_backup(fsl_ctx *ctx, const char *path, int real_bytes);
int fsl_read_backup(fsl_ctx *ctx, const char *path, int real_bytes);
/* The probe columns of Probes() (src/probes.c:21-42): stations i = LEN/2,
 * 3 LEN/4, LEN at k = DEP/2 + 1, rows j = 1..HIG, as rows[station][rho, rho u][j]
 * (6 HIG doubles). */
int fsl_probe_rows(fsl_ctx *ctx, double *rows);
/* Append one Probes() record to a probes.dat file: step, then per station HIG
 * values of rho and of rho u. */
int fsl_write_probes(fsl_ctx *ctx, const char *path, int real_bytes);
/* Favre average of the probe columns accumulated on the device, without a
 * probes file (favre-average-src/layer2_p.c:59-112): reset, accumulate the
 * current U^n, read u~[station][j] = sum(rho u) / sum(rho) and the count. */
int fsl_favre_reset(fsl_ctx *ctx);
int fsl_favre_accumulate(fsl_ctx *ctx);
int fsl_favre_read(fsl_ctx *ctx, double *u, int *count);
/* The reference's post-processor over a probes file (host only, no device):
 * records with step_start <= step <= step_end, u~[station][j] as above. */
int fsl_favre_from_probes(const char *path, int HIG, int real_bytes, int step_start, int step_end, double *u,
                          int *records);
/* The reference post-processor itself (favre-average-src/layer2_p.c:30-146,
 * host only): a probes file of float records (fsl_write_probes with
 * real_bytes 4, the reference's format), the records with step_start <= step
 * <= step_end summed in float, u~ = sum(rho u) / sum(rho) in float, written as
 * dir/probe1.dat .. dir/probe3.dat in its text format; *records (may be
 * NULL) receives the number summed.  Reading stops at the end of the file
 * (the reference's loop re-adds its last record there until killed). */
int fsl_favre_profiles(const char *path, int HIG, int step_start, int step_end, const char *dir, int *records);

/* Output() (src/output.c:16-141): per interior cell, in its loop order (k,
 * then j, then i fastest), the 12 values x, y, z, rho, u, v, w, p, T,
 * vorticity magnitude, Q criterion and rho Cs DD |S| / mu_L in the reference's
 * arithmetic, from the current U^n with the ghost layer the last stage left
 * (call after fsl_step, as the reference calls Output() after the stages).
 * fsl_output_fields fills 12 LEN HIG DEP doubles; fsl_write_tecplot writes the
 * ASCII Tecplot file; fsl_tecplot_write writes such values (host only). */
int fsl_output_fields(fsl_ctx *ctx, double *fields);
int fsl_write_tecplot(fsl_ctx *ctx, const char *path);
int fsl_tecplot_write(const char *path, int LEN, int HIG, int DEP, const double *fields);

/* ---- learned subgrid closure ---------------------------------------------------
 * No counterpart in the reference (project extension).  A per-cell MLP
 * 8 -> 64 -> 64 -> 64 -> 1 (SiLU; BF16 weights and activations, FP32
 * accumulation on the tensor cores) maps the local strain rate |S| (as
 * log(1 + |S| t_ref)), the five independent strain-rate components over |S|,
 * the density and the filter width over len_ref to the Smagorinsky
 * coefficient Cs^2; mu_SGS = rho Cs^2 (dx dy dz)^(2/3) |S| as in the dynamic
 * procedure (src/turbulence.c:442).  With params.sgs = FSL_SGS_LEARNED the
 * steps use it; every `every` steps the dynamic procedure runs beside it as the
 * judge, on the plane-averaged SGS viscosity profiles <mu>(y) of both closures
 * over the cells at least two from every boundary.  The steps fall back to the
 * dynamic procedure while either criterion fails:
 *   - effective viscosity: |<mu_mlp> - <mu_dyn>|_2 / |mu_L + <mu_dyn>|_2 over
 *     all rows exceeds `threshold` (fsl_closure_judge, default 0.05) -- what
 *     the viscous fluxes see;
 *   - SGS viscosity where the model acts: over the rows whose <mu_dyn> is at
 *     least `floor` mu_L (fsl_closure_judge_active, default floor 0.1),
 *     |<mu_mlp> - <mu_dyn>|_2 / |<mu_dyn>|_2 exceeds `threshold` (default
 *     0.4).  Where the dynamic procedure gives SGS viscosity comparable to the
 *     molecular one, a network that predicts too little (or nothing) fails
 *     here even when the first criterion, dominated by mu_L, would pass.
 * The Cs^2 errors and the SGS viscosity error relative to the dynamic SGS
 * viscosity alone are reported too; per cell the dynamic Cs^2 is dominated by
 * cell-to-cell noise, and where |S| vanishes it does not act. */
#define FSL_CLOSURE_NPARAMS 9473 /* W1[64][16] b1 W2[64][64] b2 W3[64][64] b3 w4[64] b4 */

typedef struct fsl_closure_stats {
    double profile_err;    /* last judgement: |<Cs2_mlp>(y) - <Cs2_dyn>(y)|_2 / |<Cs2_dyn>(y)|_2 */
    double cell_err;       /* last judgement: |Cs2_mlp - Cs2_dyn|_2 / |Cs2_dyn|_2 over cells */
    double mu_profile_err; /* last judgement: |<mu_mlp>(y) - <mu_dyn>(y)|_2 / |<mu_dyn>(y)|_2 */
    double visc_err;       /* last judgement: |<mu_mlp>(y) - <mu_dyn>(y)|_2 / |mu_L + <mu_dyn>(y)|_2
                              (the fallback criterion) */
    int judgements, fallbacks, using_dynamic;
    unsigned last_step;
    double mu_active_err;  /* last judgement: |<mu_mlp> - <mu_dyn>|_2 / |<mu_dyn>|_2 over the rows whose
                              <mu_dyn> >= floor mu_L (0 when there are none) */
    double dyn_ratio;      /* last judgement: max over rows of <mu_dyn>(y) / mu_L */
    int active_rows;       /* last judgement: rows in mu_active_err */
    int dynamic_steps;     /* steps whose SGS viscosity came from the dynamic procedure (fallback) */
} fsl_closure_stats;

/* Feature scales: t_ref = delta_w0 / dU (time scale of |S|), len_ref = delta_w0. */
int fsl_closure_set_scales(fsl_ctx *ctx, double t_ref, double len_ref);
int fsl_closure_set_weights(fsl_ctx *ctx, const float *params);
int fsl_closure_get_weights(fsl_ctx *ctx, float *params);
/* Judge every `every` steps (0: never) with the effective-viscosity threshold. */
int fsl_closure_judge(fsl_ctx *ctx, int every, double threshold);
/* The second criterion: rows with <mu_dyn> >= floor mu_L are judged on the
 * SGS viscosity profile itself, with `threshold` (floor > 0, threshold >= 0). */
int fsl_closure_judge_active(fsl_ctx *ctx, double floor, double threshold);
int fsl_closure_get_stats(fsl_ctx *ctx, fsl_closure_stats *stats);
/* Both closures on the current U^n: Cs^2 of the MLP and of the dynamic
 * procedure (padded FP32 host arrays, either may be NULL) and the four errors
 * of one judgement in *errs (its counters are the context's). */
int fsl_closure_compare(fsl_ctx *ctx, float *cs2_mlp, float *cs2_dyn, fsl_closure_stats *errs);

/* Training on (features, dynamic Cs^2) samples harvested on the GPU. */
typedef struct fsl_trainer fsl_trainer;
int fsl_trainer_create(long long capacity, unsigned long long seed, fsl_trainer **tr);
int fsl_trainer_destroy(fsl_trainer *tr);
/* Append every stride-th cell of ctx's U^n at least two cells from every
 * boundary, with the dynamic procedure's Cs^2 (nearer the boundary that value
 * carries the zero padding of the reference's test filter).  Judgements use
 * the same band. */
int fsl_trainer_harvest(fsl_trainer *tr, fsl_ctx *ctx, int stride);
long long fsl_trainer_size(fsl_trainer *tr);
int fsl_trainer_get_samples(fsl_trainer *tr, float *X, float *Y, long long n); /* first n: X[n][8], Y[n] */
int fsl_trainer_set_samples(fsl_trainer *tr, const float *X, const float *Y, long long n);
int fsl_trainer_get_weights(fsl_trainer *tr, float *params);
int fsl_trainer_set_weights(fsl_trainer *tr, const float *params);
/* Loss: 0 = mean squared error of Cs^2; 1 (default) = each sample weighted by
 * (rho |S| t_ref)^2 over the mean weight of all samples, i.e. the squared
 * error of mu_SGS = rho Cs^2 DD |S| the closure feeds into the fluxes. */
int fsl_trainer_set_loss(fsl_trainer *tr, int mode);
/* Loss gradient over the first n samples at the current weights. */
int fsl_trainer_gradient(fsl_trainer *tr, long long n, float *grad, double *loss);
/* Adam on shuffled mini-batches; *loss receives the final full-set MSE. */
int fsl_trainer_train(fsl_trainer *tr, int epochs, long long batch, double lr, double *loss);

/* ---- ensembles -------------------------------------------------------------
 * No counterpart in the reference (project extension; the reference runs one
 * domain per process).  Independent temporal shear layers -- each an ordinary
 * context with its own grid, Mach number, Reynolds number and seed -- advance
 * together: fsl_ensemble_step captures `chunk` fused steps of every member
 * (each on its own stream, forked from and joined to the ensemble's stream)
 * into one CUDA graph and replays it, so the members' kernels share the SMs
 * and a chunk costs one launch.  Every member's result is bit-identical to
 * stepping it alone with fsl_step.  Members: temporal setup, nStages = 3,
 * either reconstruction, whole domains (not x-slabs), no profiling, learned
 * closure only with judgements off
 * (fsl_closure_judge(ctx, 0, ...)); otherwise FSL_ERR_UNSUPPORTED.  A member
 * in the middle of a stage-wise step (fsl_step_stage) is refused with
 * FSL_ERR_ARG.  Members stay owned by the caller and must outlive the ensemble; while an ensemble
 * step is in flight, do not call them directly.  Each member's disturbance
 * RNG state (unused by the temporal setup) is not advanced by replays. */
typedef struct fsl_ensemble fsl_ensemble;
int fsl_ensemble_create(fsl_ctx *const *members, int n, fsl_ensemble **ens);
int fsl_ensemble_destroy(fsl_ensemble *ens);
const char *fsl_ensemble_last_error(const fsl_ensemble *ens);
/* The ensemble's CUDA stream (cudaStream_t); its work follows and precedes
 * the members' own streams. */
void *fsl_ensemble_stream(fsl_ensemble *ens);
/* Steps captured per graph (1..1000, default 10). */
int fsl_ensemble_set_chunk(fsl_ensemble *ens, int steps);
int fsl_ensemble_step(fsl_ensemble *ens, int nsteps);
int fsl_ensemble_sync(fsl_ensemble *ens);
/* 1 when the ensemble steps on the persistent path: all members FP32 bulk,
 * reference reconstruction, full-lane tiles (FSL_TUNE_STAGE_ROWS 0).  A step
 * is then the members' work before their first stage, each on its own
 * stream, and ONE cooperative launch that runs the three stages of every
 * member, balanced over one block per SM, with grid barriers between the
 * stages (where the blocks also fill the new states' ghost layers and
 * boundary faces).  A member keeps the split of its planes into blocks that
 * its own launches use, so its results are bit-identical to stepping it
 * alone.  0: each member's fused steps, replayed from a CUDA graph. */
int fsl_ensemble_persistent(fsl_ensemble *e);
/* Polls (64 ns sleeps) a grid barrier of the persistent launch waits for the
 * other blocks before it gives up (default 2^24).  A barrier that gives up
 * ends the launch early and fsl_ensemble_sync returns FSL_ERR_TIMEOUT; the
 * members' states of that step are then incomplete (upload them again). */
int fsl_ensemble_set_barrier_limit(fsl_ensemble *e, unsigned polls);
/* Autotuner of the fused-stage tile shape (tile rows 8/12/16 x planes per
 * block 8/16/32/64, one shape for all members): each candidate is timed on
 * the device over one graph replay of trial_steps ensemble steps; the
 * fastest is kept and every member's state, time step and counters are
 * restored, so tuning changes no result. */
int fsl_ensemble_tune(fsl_ensemble *ens, int trial_steps, int *rows, int *seg, double *ms_per_step);

/* ---- profiling ------------------------------------------------------------- */

/* Kernel classes timed by the context's profiler. */
#define FSL_K_STAGE 0 /* fused stage kernel */
#define FSL_K_RECON 1 /* per-phase reconstruction */
#define FSL_K_FLUX 2  /* per-phase fluxes */
#define FSL_K_SGS 3   /* SGS viscosity (dynamic procedure or learned closure) */
#define FSL_K_EVOL 4  /* per-phase RK update */
#define FSL_K_BC 5    /* ghost cells and boundary faces */
#define FSL_K_CFL 6   /* Courant reduction and dt rescale */
#define FSL_K_OTHER 7 /* state transfer, diagnostics */
#define FSL_K_COUNT 8

typedef struct fsl_ktimes {
    double ms[FSL_K_COUNT];                  /* device time per class (CUDA events on the context stream) */
    unsigned long long launches[FSL_K_COUNT]; /* kernels launched per class */
} fsl_ktimes;

/* Reset the counters; with on != 0, bracket every kernel class with CUDA
 * events from now on (launch counts are always kept). */
int fsl_profile(fsl_ctx *ctx, int on);
/* Synchronise and read the accumulated times and launch counts. */
int fsl_profile_read(fsl_ctx *ctx, fsl_ktimes *out);
/* The CUDA stream (cudaStream_t) all work of the context runs on. */
void *fsl_stream(fsl_ctx *ctx);

/* ---- diagnostics ----------------------------------------------------------- */

/* Both over the planes of the Courant range (fsl_set_courant_range): the
 * whole interior, or an x-slab's owned planes, whose results add up across
 * the slabs (the SUM all-reduce of the distributed variant's integrals). */
/* Volume integrals of rho, rho u, rho v, rho w, E over the interior (FP64). */
int fsl_sums(fsl_ctx *ctx, double sums[5]);
/* Per y-row sums over the interior x-z plane of rho, rho u, rho v, rho w,
 * rho uu, rho vv, rho ww, rho uv (rows[8*HIG], FP64). */
int fsl_plane_sums(fsl_ctx *ctx, double *rows);

#ifdef __cplusplus
}
#endif
#endif /* FSL_GPU_H */
