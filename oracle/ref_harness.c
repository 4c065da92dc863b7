/*
 * ref_harness.c -- test-only driver around the reference's serial solver.
 *
 * Linked with the reference's own src/ C files (compiled in place, FP64 + zero-fill
 * patch, main renamed ref_main) into oracle/_ref/libfslref.so.  It gives the
 * tests per-phase access to the reference's global state (src/global.h:6-72)
 * so that every phase of the explicit step can be checked in isolation:
 * set arrays and scalars, call one reference phase, read the arrays back.
 *
 * Nothing here re-implements reference arithmetic: the phase entry points call
 * the reference functions directly.  refh_step() restates only the control
 * flow of the driver loop body (src/layer2.c:141-185) without its I/O
 * (Probes/Output), so that N-step runs can be compared.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "type.h"
#include "def.h"
#include "global.h"
#include "helpers.h"
#include "turbulence.h"
#include "reconstruction.h"

void Initialize(void);
void BounCondInGhostCells(void);
void Reconstruction(void);
void BounCondOnInterfaces(void);
void Fluxes(void);
void Evolution(int numStages, int Stage);

/* the driver's block-period counter (a local of main() at src/layer2.c:120) */
static int refh_counter = 0;

/* src/fluxes.c compiled a second time with its static Smagorinsky branch
 * live (DynamicSmagorinskySGS 0, as src-par/def.h:47 sets it; see
 * ref_static.h).  refh_set_static(1) makes refh_step use it. */
void Fluxes_static(void);
static int refh_static = 0;
void refh_set_static(int on) { refh_static = on; }

/* Run Initialize() (src/initialize.c:14-192) with `dir` as the working
 * directory, so that it reads dir/layer2.ini (and dir/backup.dat on restart). */
int refh_init(const char *dir)
{
    char saved[4096];
    if (!getcwd(saved, sizeof saved)) return -1;
    if (chdir(dir) != 0) return -2;
    Initialize();
    if (chdir(saved) != 0) return -3;
    refh_counter = 0;
    return 0;
}

void refh_seed(double x) { X = x; refh_counter = 0; }

/* Disturbance draw of the driver loop, src/layer2.c:152-162 (printing removed). */
void refh_disturb(void)
{
    if (refh_counter > 0) refh_counter--;
    else {
        refh_counter = (int)(Ns_min + Nst * (X = Random(X)));
        k_min = (unsigned)(DEP * (X = Random(X)));
        k_max = (unsigned)(k_min + DEP * (X = Random(X)));
        if (k_max > DEP) k_max -= DEP;
        X = Random(X); Ud = Ua * (1 - X - X);
        X = Random(X); Vd = Va * (1 - X - X);
        X = Random(X); Wd = Wa * (1 - X - X);
    }
}

/* n iterations of the driver loop body, src/layer2.c:141-185, without I/O. */
void refh_step(int n)
{
    int s;
    while (n-- > 0) {
        checkCoNum();
        ++step;
        refh_disturb();
        for (s = 1; s <= nStages; s++) {
            Stage = (char)s;
            BounCondInGhostCells();
            Reconstruction();
            BounCondOnInterfaces();
            if (refh_static) Fluxes_static();
            else Fluxes();
            Evolution(nStages, s);
        }
    }
}

void refh_ghost(void) { BounCondInGhostCells(); }
void refh_recon(void) { Reconstruction(); }
void refh_ifbc(void) { BounCondOnInterfaces(); }
void refh_fluxes(void) { Fluxes(); }
void refh_fluxes_static(void) { Fluxes_static(); }
void refh_evolution(int nst, int stage) { Evolution(nst, stage); }
void refh_dynsmag(void) { DynamicSmagorinsky(U1, U2, U3, U4, mu_SGS); }
void refh_checkco(void) { checkCoNum(); }
/* Output() writes "<step>.plt" into `dir` (src/output.c:16-141); its header
 * file declares nothing. */
void Output(void);
int refh_output(const char *dir)
{
    char saved[4096];
    if (!getcwd(saved, sizeof saved)) return -1;
    if (chdir(dir) != 0) return -2;
    Output();
    if (chdir(saved) != 0) return -3;
    return 0;
}

/* ---- array access ---------------------------------------------------- */

static real ***cell_array(int which, int var)
{
    real ***u[5], ***up[5], ***cur[5];
    u[0] = U1; u[1] = U2; u[2] = U3; u[3] = U4; u[4] = U5;
    up[0] = U1p; up[1] = U2p; up[2] = U3p; up[3] = U4p; up[4] = U5p;
    cur[0] = U1_; cur[1] = U2_; cur[2] = U3_; cur[3] = U4_; cur[4] = U5_;
    if (var < 0 || var > 4) return NULL;
    switch (which) {
    case 0: return u[var];
    case 1: return up[var];
    case 2: return cur[var];
    case 3: return mu_SGS;
    default: return NULL;
    }
}

/* which: 0 = U^n (U1..U5), 1 = stage buffer (U1p..U5p), 2 = current-stage
 * pointers (U1_..U5_), 3 = mu_SGS (var ignored).  Layout of `buf`: padded
 * (LEN+2)(HIG+2)(DEP+2), k fastest. */
int refh_cells(int which, int var, double *buf, int write)
{
    unsigned a, b, c;
    size_t n = 0;
    real ***p = cell_array(which, which == 3 ? 0 : var);
    if (!p) return -1;
    for (a = 0; a < LEN + 2; a++)
        for (b = 0; b < HIG + 2; b++)
            for (c = 0; c < DEP + 2; c++, n++) {
                if (write) p[a][b][c] = buf[n];
                else buf[n] = p[a][b][c];
            }
    return 0;
}

/* dir 0/1/2 = x/y/z faces; side 0 = the minus-side state array (xU*, yU*,
 * zU*; holds the flux after Fluxes()), side 1 = the plus-side state array
 * (U*x, U*y, U*z).  Layout: dense over the reference's face index ranges,
 * x: (LEN+1)*HIG*DEP, y: LEN*(HIG+1)*DEP, z: LEN*HIG*(DEP+1). */
int refh_faces(int dir, int side, int var, double *buf, int write)
{
    real ***tab[3][2][5] = {
        {{xU1, xU2, xU3, xU4, xU5}, {U1x, U2x, U3x, U4x, U5x}},
        {{yU1, yU2, yU3, yU4, yU5}, {U1y, U2y, U3y, U4y, U5y}},
        {{zU1, zU2, zU3, zU4, zU5}, {U1z, U2z, U3z, U4z, U5z}},
    };
    unsigned na, nb, nc, a, b, c;
    size_t n = 0;
    real ***p;
    if (dir < 0 || dir > 2 || side < 0 || side > 1 || var < 0 || var > 4) return -1;
    p = tab[dir][side][var];
    na = LEN + (dir == 0); nb = HIG + (dir == 1); nc = DEP + (dir == 2);
    for (a = 0; a < na; a++)
        for (b = 0; b < nb; b++)
            for (c = 0; c < nc; c++, n++) {
                if (write) p[a][b][c] = buf[n];
                else buf[n] = p[a][b][c];
            }
    return 0;
}

/* Point U*_ at U (0) or at the stage buffer U*p (1). */
void refh_set_cur(int which)
{
    if (which == 0) { U1_ = U1; U2_ = U2; U3_ = U3; U4_ = U4; U5_ = U5; }
    else { U1_ = U1p; U2_ = U2p; U3_ = U3p; U4_ = U4p; U5_ = U5p; }
}
int refh_get_cur(void) { return U1_ == U1 ? 0 : 1; }

/* Scalars in a fixed order, as doubles:
 * 0 deltaT 1 deltaT_X 2 deltaT_Y 3 deltaT_Z 4 X 5 k_min 6 k_max 7 Ud 8 Vd
 * 9 Wd 10 step 11 DD 12 lambda_L 13 cp_Pr_T 14 maxCoNum 15 counter */
void refh_get_scalars(double *o)
{
    o[0] = deltaT; o[1] = deltaT_X; o[2] = deltaT_Y; o[3] = deltaT_Z;
    o[4] = X; o[5] = k_min; o[6] = k_max; o[7] = Ud; o[8] = Vd; o[9] = Wd;
    o[10] = step; o[11] = DD; o[12] = lambda_L; o[13] = cp_Pr_T;
    o[14] = maxCoNum; o[15] = refh_counter;
}

/* Set the time step the way checkCoNum() leaves it (src/helpers.c:47-50). */
void refh_set_dt(double dt)
{
    deltaT = dt;
    deltaT_X = deltaT / deltaX; deltaT_Y = deltaT / deltaY; deltaT_Z = deltaT / deltaZ;
}

void refh_set_disturbance(unsigned kmin, unsigned kmax, double ud, double vd, double wd)
{
    k_min = kmin; k_max = kmax; Ud = ud; Vd = vd; Wd = wd;
}

/* Test filter of one padded field through the reference's filter_()
 * (src/turbulence.c:17-100) with the box kernel used at :113. */
int refh_filter(const double *in, double *out)
{
    real h[3] = {1. / 3., 1. / 3., 1. / 3.};
    real ***a = Array3D(LEN + 2, HIG + 2, DEP + 2), ***f;
    unsigned x, y, z;
    size_t n = 0;
    for (x = 0; x < LEN + 2; x++)
        for (y = 0; y < HIG + 2; y++)
            for (z = 0; z < DEP + 2; z++) a[x][y][z] = in[n++];
    f = filter_(a, h);
    n = 0;
    for (x = 0; x < LEN + 2; x++)
        for (y = 0; y < HIG + 2; y++)
            for (z = 0; z < DEP + 2; z++) out[n++] = f[x][y][z];
    free3D(a, LEN + 2, HIG + 2);
    free3D(f, LEN + 2, HIG + 2);
    return 0;
}

double refh_minmod(double x, double y) { return minmod(x, y); }
double refh_random(double x) { return Random(x); }
