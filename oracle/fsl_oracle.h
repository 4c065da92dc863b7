/*
 * fsl_oracle.h -- CPU restatement of freeShearLayer's explicit time step.
 *
 * TEST INFRASTRUCTURE ONLY.  The product (freeshearlayer_b200) never links,
 * includes or calls this code; tests, the smoke check and the CPU-baseline leg
 * of the benchmark use it as the checker.
 *
 * Parity pin: on the reference spatial case every phase of this restatement
 * is compared bit-for-bit with the reference's own serial solver (src/),
 * compiled in place with the FP64 + zero-fill oracle patch into
 * oracle/_ref/libfslref.so (tests/test_oracle_vs_ref.py), and with committed
 * golden vectors generated from it (tests/golden/).  The temporal shear-layer
 * setup (periodic x, zero-gradient y) exists only in this project; those
 * boundary rules are pinned by this restatement alone.
 *
 * Arithmetic is FP64 with every expression evaluated in the reference's
 * order; build with -ffp-contract=off.
 *
 * Layout: cell arrays are padded (LEN+2)(HIG+2)(DEP+2), k fastest, like the
 * reference's Array3D(LEN+2,HIG+2,DEP+2) (src/helpers.c:58-80) flattened.
 * Face arrays are dense over the reference's face index ranges:
 *   x: (LEN+1)*HIG*DEP, y: LEN*(HIG+1)*DEP, z: LEN*HIG*(DEP+1).
 */
#ifndef FSL_ORACLE_H
#define FSL_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SETUP_SPATIAL = 0, ORC_SETUP_TEMPORAL = 1 };
enum { ORC_CFL_STREAMWISE = 0, ORC_CFL_ACOUSTIC = 1 };

typedef struct orc_params {
    /* the 22 positional values of layer2.ini (src/initialize.c:25-58) */
    int LEN, HIG, DEP;
    double deltaX, deltaY, deltaZ, deltaT;
    int Answer, numstep;
    double mu_L, Pr_L, Pr_T, Cs;
    int BL_HIG;
    double Ua, Va, Wa;
    int Ns_min, Nst, f_step, nStages;
    double maxCoNum;
    /* project extensions */
    int setup;     /* ORC_SETUP_* */
    int cfl_mode;  /* ORC_CFL_* */
    double seed_X; /* disturbance RNG seed (the reference reads it from stdin) */
    int recon;     /* 0: the reference's reconstruction, 1: PPM (project extension) */
    int sgs;       /* ORC_SGS_*: the SGS viscosity the face fluxes use */
} orc_params;

/* SGS models (values as FSL_SGS_* of the product's C ABI).  DYNAMIC is the
 * reference's hardcoded choice (src/def.h:47, DynamicSmagorinskySGS 1);
 * STATIC is its other branch, rho_face Cs DD |S|_face per face
 * (src/fluxes.c:193-205, :362-374, :533-545), live in src-par/def.h:47;
 * NONE sets the SGS viscosity to zero. */
enum { ORC_SGS_DYNAMIC = 0, ORC_SGS_STATIC = 2, ORC_SGS_NONE = 3 };

typedef struct orc_ctx orc_ctx;

orc_ctx *orc_create(const orc_params *p);
void orc_destroy(orc_ctx *o);

/* state access.  which: 0 = U^n, 1 = stage buffer Up, 2 = current-stage
 * pointer (U*_), 3 = mu_SGS (var ignored).  Padded layout. */
int orc_cells(orc_ctx *o, int which, int var, double *buf, int write);
/* face arrays; side 0 = minus state / flux (xU*), side 1 = plus state (U*x) */
int orc_faces(orc_ctx *o, int dir, int side, int var, double *buf, int write);
/* interior state in the backup.dat row layout (src/finalize.c:22-29):
 * for i, for j: DEP values of U1, then U2 .. U5.  Writes/reads U^n. */
int orc_state(orc_ctx *o, double *buf, int write);
void orc_set_cur(orc_ctx *o, int which);
int orc_get_cur(orc_ctx *o);

/* scalars, same order as the reference harness: 0 deltaT 1 dtx 2 dty 3 dtz
 * 4 X 5 k_min 6 k_max 7 Ud 8 Vd 9 Wd 10 step 11 DD 12 lambda_L 13 cp_Pr_T
 * 14 maxCoNum 15 counter 16 last maxCo */
void orc_get_scalars(orc_ctx *o, double *out);
void orc_set_dt(orc_ctx *o, double dt);
void orc_set_disturbance(orc_ctx *o, unsigned kmin, unsigned kmax, double ud, double vd, double wd);

/* phases (reference names in comments) */
void orc_ghost_bc(orc_ctx *o);          /* BounCondInGhostCells */
void orc_reconstruct(orc_ctx *o);       /* Reconstruction */
void orc_interface_bc(orc_ctx *o);      /* BounCondOnInterfaces */
void orc_dynamic_smagorinsky(orc_ctx *o); /* DynamicSmagorinsky(U1..U4, mu_SGS) */
void orc_fluxes_only(orc_ctx *o);       /* Fluxes() without the SGS call */
void orc_fluxes(orc_ctx *o);            /* Fluxes() including the SGS call */
void orc_evolution(orc_ctx *o, int nstages, int stage); /* Evolution */
double orc_check_courant(orc_ctx *o);   /* checkCoNum; returns maxCo */
void orc_disturb(orc_ctx *o);           /* driver's block draw */
void orc_step(orc_ctx *o, int nsteps);  /* driver loop body, SGS once per step */
void orc_step_ref_sgs(orc_ctx *o, int nsteps); /* same, SGS recomputed every stage */

/* standalone pieces */
void orc_filter(const orc_params *p, const double *in, double *out);
double orc_minmod(double x, double y);
double orc_random(double x);

/* temporal shear layer initial state (project extension); interior state in
 * the backup.dat layout.  Returns dU (velocity difference) in *dU_out. */
int orc_temporal_state(const orc_params *p, double Mc, double delta_w0, double amp,
                       unsigned long long seed, double *state, double *dU_out);

/* diagnostics (project extension), FP64 over U^n.
 * sums[5]: volume integrals of the conserved variables.
 * rows[8*HIG]: per y-row plane sums of rho, rho u, rho v, rho w, rho uu,
 * rho vv, rho ww, rho uv over the interior x-z plane. */
void orc_sums(orc_ctx *o, double *sums);
void orc_plane_sums(orc_ctx *o, double *rows);
/* Output()'s 12 values per cell, src/output.c:66-139 (k, j, i order). */
void orc_output_fields(orc_ctx *o, double *out);

#ifdef __cplusplus
}
#endif
#endif
