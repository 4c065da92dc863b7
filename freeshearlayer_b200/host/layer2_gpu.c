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
 * and from an optional ./layer2_gpu.ini beside layer2.ini (which stays the
 * reference's 22 positional lines), one `key = value` per line, `#` starting
 * a comment:
 *   precision = fp64 | fp32          arithmetic of the step (FSL_PREC_*)
 *   sgs = dynamic | learned | static | none   subgrid model (FSL_SGS_*)
 *   recon = minmod | ppm             reconstruction (FSL_RECON_*)
 *   setup = spatial | temporal       boundary setup (as FSL_SETUP)
 *   cfl = streamwise | acoustic      Courant number (as FSL_CFL)
 *   closure_weights = <path>         learned closure: FSL_CLOSURE_NPARAMS
 *                                    little-endian float32 parameters
 *   closure_t_ref = <s>              its feature scales: delta_w0 / dU ...
 *   closure_len_ref = <m>            ... and delta_w0
 *   judge_every = <steps>            dynamic-procedure judgements (0: none)
 *   judge_threshold = <x>            effective-viscosity criterion
 *   temporal_state = <Mc> <delta_w0> <amp> <seed>   fresh start from the
 *                                    temporal shear layer instead of the
 *                                    reference's inflow profile
 */
#include <signal.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fsl_gpu.h"

static volatile sig_atomic_t contin_flag = 1;

/* The options of ./layer2_gpu.ini (all optional). */
struct gpu_opts {
    char weights[256];
    double t_ref, len_ref, judge_thr;
    int judge_every;
    int temporal;
    double Mc, dw0, amp;
    unsigned long long seed;
};

static int word_is(const char *a, const char *b) { return strcmp(a, b) == 0; }

/* Read ./layer2_gpu.ini into p and o; 0 when it is absent or read, -1 on a
 * line it does not understand. */
static int read_gpu_ini(fsl_params *p, struct gpu_opts *o)
{
    char line[512], key[64], val[256];
    FILE *f = fopen("layer2_gpu.ini", "r");
    int lineno = 0;
    if (!f) return 0;
    while (fgets(line, sizeof line, f)) {
        char *hash = strchr(line, '#');
        lineno++;
        if (hash) *hash = '\0';
        key[0] = val[0] = '\0';
        if (sscanf(line, " %63[A-Za-z_] = %255[^\n]", key, val) < 1) continue; /* blank line */
        {
            size_t m = strlen(val); /* trailing blanks and a CR */
            while (m > 0 && (val[m - 1] == ' ' || val[m - 1] == '\t' || val[m - 1] == '\r')) val[--m] = '\0';
        }
        if (word_is(key, "precision") && (word_is(val, "fp64") || word_is(val, "fp32")))
            p->precision = word_is(val, "fp32") ? FSL_PREC_FP32 : FSL_PREC_FP64;
        else if (word_is(key, "sgs") && word_is(val, "dynamic")) p->sgs = FSL_SGS_DYNAMIC;
        else if (word_is(key, "sgs") && word_is(val, "learned")) p->sgs = FSL_SGS_LEARNED;
        else if (word_is(key, "sgs") && word_is(val, "static")) p->sgs = FSL_SGS_STATIC;
        else if (word_is(key, "sgs") && word_is(val, "none")) p->sgs = FSL_SGS_NONE;
        else if (word_is(key, "recon") && (word_is(val, "minmod") || word_is(val, "ppm")))
            p->recon = word_is(val, "ppm") ? FSL_RECON_PPM : FSL_RECON_CHARMINMOD;
        else if (word_is(key, "setup") && (word_is(val, "spatial") || word_is(val, "temporal")))
            p->setup = word_is(val, "temporal") ? FSL_SETUP_TEMPORAL : FSL_SETUP_SPATIAL;
        else if (word_is(key, "cfl") && (word_is(val, "streamwise") || word_is(val, "acoustic")))
            p->cfl_mode = word_is(val, "acoustic") ? FSL_CFL_ACOUSTIC : FSL_CFL_STREAMWISE;
        else if (word_is(key, "closure_weights") && sscanf(val, "%255s", o->weights) == 1) ;
        else if (word_is(key, "closure_t_ref") && sscanf(val, "%lf", &o->t_ref) == 1) ;
        else if (word_is(key, "closure_len_ref") && sscanf(val, "%lf", &o->len_ref) == 1) ;
        else if (word_is(key, "judge_every") && sscanf(val, "%d", &o->judge_every) == 1) ;
        else if (word_is(key, "judge_threshold") && sscanf(val, "%lf", &o->judge_thr) == 1) ;
        else if (word_is(key, "temporal_state") &&
                 sscanf(val, "%lf %lf %lf %llu", &o->Mc, &o->dw0, &o->amp, &o->seed) == 4)
            o->temporal = 1;
        else {
            printf("layer2_gpu.ini:%d: cannot read \"%s\"\n", lineno, key);
            fclose(f);
            return -1;
        }
    }
    fclose(f);
    return 0;
}

/* The learned closure's parameters from a file of FSL_CLOSURE_NPARAMS floats. */
static int load_weights(fsl_ctx *ctx, const struct gpu_opts *o)
{
    float *w = (float *)malloc(FSL_CLOSURE_NPARAMS * sizeof(float));
    FILE *f = fopen(o->weights, "rb");
    size_t got = 0;
    int rc;
    if (!w || !f) {
        printf("Cannot open closure weights \"%s\"\n", o->weights);
        if (f) fclose(f);
        free(w);
        return -1;
    }
    got = fread(w, sizeof(float), FSL_CLOSURE_NPARAMS, f);
    fclose(f);
    if (got != FSL_CLOSURE_NPARAMS) {
        printf("closure weights \"%s\": %lu of %d values\n", o->weights, (unsigned long)got, FSL_CLOSURE_NPARAMS);
        free(w);
        return -1;
    }
    rc = (o->t_ref > 0 && o->len_ref > 0) ? fsl_closure_set_scales(ctx, o->t_ref, o->len_ref) : FSL_OK;
    if (rc == FSL_OK) rc = fsl_closure_set_weights(ctx, w);
    if (rc == FSL_OK && o->judge_every >= 0) rc = fsl_closure_judge(ctx, o->judge_every, o->judge_thr);
    free(w);
    return rc;
}

static void term_handler(int sig)
{
    (void)sig;
    contin_flag = 0;
}

int main(void)
{
    fsl_params p;
    struct gpu_opts opt;
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
    memset(&opt, 0, sizeof opt);
    opt.judge_every = -1; /* the library's default unless the file sets it */
    opt.judge_thr = 0.02;
    if (read_gpu_ini(&p, &opt) != 0) return 1;
    if (p.sgs == FSL_SGS_LEARNED && !opt.weights[0]) {
        puts("layer2_gpu.ini: sgs = learned needs closure_weights");
        return 1;
    }

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
        if (opt.temporal) fsl_temporal_state(&p, opt.Mc, opt.dw0, opt.amp, opt.seed, state, NULL);
        else fsl_initial_state(&p, state);
        fsl_upload_state(ctx, state);
    }
    if (opt.weights[0] && load_weights(ctx, &opt) != FSL_OK) {
        free(state);
        fsl_destroy(ctx);
        return 1;
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
