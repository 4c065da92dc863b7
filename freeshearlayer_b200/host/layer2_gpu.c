/*
 * layer2_gpu.c -- ANSI C driver of the B200 explicit step.
 *
 * Drop-in for the reference's driver (src/layer2.c:117-195): reads
 * ./layer2.ini, the disturbance seed from stdin, runs `numstep` steps with
 * SIGINT as a clean stop, and writes ./backup.dat in the reference's layout
 * (src/finalize.c:14-35).  A restart (Answer = 1) reads ./backup.dat the way
 * src/initialize.c:133-158 intends (fields, deltaT, step).  All arithmetic
 * runs on the GPU through libfsl_gpu (include/fsl_gpu.h); this file only
 * sequences calls and does file I/O.
 *
 * Every step appends a Probes() record to ./probes.dat (src/probes.c), every
 * f_step steps and at the end it writes the Tecplot frame <step>.plt
 * (src/output.c), as the reference's loop does (src/layer2.c:180-189).
 * Binary files are written in FP64.
 *
 * Options beyond layer2.ini come from the environment:
 *   FSL_SETUP=temporal  periodic-x temporal shear layer (default: spatial)
 *   FSL_CFL=acoustic    acoustic Courant number (default: streamwise)
 *   FSL_PHASED=1        run the per-phase kernels instead of the fused step
 *   FSL_PROBES=0        no probes.dat records
 *   FSL_FRAMES=0        no Tecplot frames
 */
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fsl_gpu.h"

static volatile sig_atomic_t contin_flag = 1;

static void term_handler(int sig)
{
    (void)sig;
    contin_flag = 0;
}

int main(void)
{
    fsl_params p;
    fsl_ctx *ctx = NULL;
    fsl_info info;
    double *state;
    double X;
    const char *env;
    int rc, phased, probes, frames;
    char frame[64];
    size_t n;

    signal(SIGINT, term_handler);
    fsl_params_default(&p);
    if (fsl_params_from_ini("layer2.ini", &p) != FSL_OK) {
        printf("Cannot open \"layer2.ini\" file\n");
        return 1;
    }
    if (scanf("%lf", &X) == 1) {
        printf("Random number [0...1]: X = %f\n", X);
        p.seed_X = X;
    } else {
        printf("Failed to read random number.\n");
    }
    env = getenv("FSL_SETUP");
    if (env && strcmp(env, "temporal") == 0) p.setup = FSL_SETUP_TEMPORAL;
    env = getenv("FSL_CFL");
    if (env && strcmp(env, "acoustic") == 0) p.cfl_mode = FSL_CFL_ACOUSTIC;
    env = getenv("FSL_PHASED");
    phased = env && atoi(env) != 0;
    env = getenv("FSL_PROBES");
    probes = !env || atoi(env) != 0;
    env = getenv("FSL_FRAMES");
    frames = !env || atoi(env) != 0;

    printf("Total number of cells in computational domain: %d\n", p.LEN * p.HIG * p.DEP);
    rc = fsl_init(&p, &ctx);
    if (rc != FSL_OK) {
        printf("fsl_init failed: %d\n", rc);
        return 1;
    }
    n = (size_t)p.LEN * p.HIG * 5 * p.DEP;
    state = (double *)malloc(n * sizeof(double));
    if (!state) {
        puts("Cannot allocate memory");
        fsl_destroy(ctx);
        return 1;
    }
    if (p.Answer) {
        if (fsl_read_backup(ctx, "backup.dat", 8) != FSL_OK) {
            printf("Cannot read \"backup.dat\": %s\n", fsl_last_error(ctx));
            free(state);
            fsl_destroy(ctx);
            return 1;
        }
    } else {
        fsl_initial_state(&p, state);
        fsl_upload_state(ctx, state);
    }

    for (;;) {
        fsl_get_info(ctx, &info);
        if (info.step >= (unsigned)p.numstep || !contin_flag) break;
        rc = phased ? fsl_step_phased(ctx, 1) : fsl_step(ctx, 1);
        if (rc == FSL_OK) rc = fsl_sync(ctx);
        if (rc != FSL_OK) {
            printf("step failed: %d (%s)\n", rc, fsl_last_error(ctx));
            break;
        }
        fsl_get_info(ctx, &info);
        printf("Timestep no.: %u, Courant max = %f, time step = %g sec.\n", info.step, info.maxCo, info.deltaT);
        if (probes && fsl_write_probes(ctx, "probes.dat", 8) != FSL_OK)
            puts("Cannot open probes file ");
        if (frames && p.f_step > 0 && info.step % (unsigned)p.f_step == 0) {
            sprintf(frame, "%u.plt", info.step);
            if (fsl_write_tecplot(ctx, frame) != FSL_OK) fprintf(stderr, "cannot open file \"Tecplot-file\"\n");
        }
    }
    fsl_get_info(ctx, &info);
    if (frames) {
        sprintf(frame, "%u.plt", info.step);
        if (fsl_write_tecplot(ctx, frame) != FSL_OK) fprintf(stderr, "cannot open file \"Tecplot-file\"\n");
    }

    if (fsl_write_backup(ctx, "backup.dat", 8) != FSL_OK)
        puts("Cannot open \"backup.dat\" file to write");
    free(state);
    fsl_destroy(ctx);
    puts("Simulation finished!");
    return rc == FSL_OK ? 0 : 1;
}
