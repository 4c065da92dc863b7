// fsl_api.cu -- C ABI of libfsl_gpu.so (declared in include/fsl_gpu.h).
//
// Host side of the explicit step: parameter parsing (layer2.ini / .bin),
// device allocation, state transfer, the driver's per-step scalar work
// (Courant rescale, disturbance RNG) and the launch sequences.  All device
// work of a context is issued on its own CUDA stream.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>

#include "fsl_check.cuh"
#include "fsl_internal.h"

using namespace fsl;


namespace fsl {

Grid make_grid(int L, int H, int D, int elem_bytes)
{
    Grid g;
    g.L = L; g.H = H; g.D = D;
    const int q = 32 / elem_bytes; // elements per 32-byte sector
    g.pk = ((D + 2 + q - 1) / q) * q;
    g.pi = (long long)g.pk * (H + 2);
    g.off = q - 1;
    const long long n = g.off + (long long)(L + 2) * g.pi;
    g.fstride = ((n + 63) / 64) * 64;
    return g;
}

static cudaEvent_t take_event(Ctx &c)
{
    if (!c.evpool.empty()) {
        cudaEvent_t e = c.evpool.back();
        c.evpool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(Ctx &c, int cls)
{
    if (!c.prof) return;
    c.open_cls = cls;
    c.open_ev = take_event(c);
    cudaEventRecord(c.open_ev, c.stream);
}

void prof_end(Ctx &c, int cls, int nkernels)
{
    c.klaunch[cls] += (unsigned long long)nkernels;
    if (!c.prof || c.open_cls != cls || !c.open_ev) return;
    cudaEvent_t b = take_event(c);
    cudaEventRecord(b, c.stream);
    c.recs.push_back({cls, c.open_ev, b});
    c.open_ev = nullptr;
    c.open_cls = -1;
}

} // namespace fsl

namespace {

const char *kNoCtx = "no context";

int fail(Ctx &c, int code, const char *what, cudaError_t e = cudaSuccess)
{
    char buf[512];
    if (e != cudaSuccess) snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    else snprintf(buf, sizeof buf, "%s", what);
    c.err = buf;
    return code;
}

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) return fail(c, FSL_ERR_CUDA, #call, e_);            \
    } while (0)

#define CKL()                                                                      \
    do {                                                                           \
        cudaError_t e_ = cudaGetLastError();                                       \
        if (e_ != cudaSuccess) return fail(c, FSL_ERR_CUDA, "kernel launch", e_); \
    } while (0)

int dev_alloc(Ctx &c, double **p, size_t n)
{
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(double));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, FSL_ERR_NOMEM, "cudaMalloc", e);
    }
    c.bytes += n * sizeof(double);
    e = cudaMemsetAsync(*p, 0, n * sizeof(double), c.stream);
    if (e != cudaSuccess) return fail(c, FSL_ERR_CUDA, "cudaMemsetAsync", e);
    return FSL_OK;
}

size_t face_count(const Grid &g, int d)
{
    return (size_t)(g.L + (d == 0)) * (g.H + (d == 1)) * (g.D + (d == 2));
}

int ensure_faces(Ctx &c)
{
    if (c.faces_alloc) return FSL_OK;
    for (int d = 0; d < 3; d++)
        for (int s = 0; s < 2; s++)
            for (int v = 0; v < 5; v++) {
                double *p;
                int rc = dev_alloc(c, &p, face_count(c.g, d));
                if (rc) return rc;
                if (d == 0) c.f.x[s][v] = p;
                else if (d == 1) c.f.y[s][v] = p;
                else c.f.z[s][v] = p;
            }
    c.faces_alloc = true;
    return FSL_OK;
}

int ensure_dyn(Ctx &c)
{
    if (c.dyn_alloc) return FSL_OK;
    const size_t fs = (size_t)c.g.fstride;
    int rc;
    if ((rc = dev_alloc(c, &c.dyn.vel, 3 * fs))) return rc;
    if ((rc = dev_alloc(c, &c.dyn.F, 9 * fs))) return rc;
    if ((rc = dev_alloc(c, &c.dyn.A, 6 * fs))) return rc;
    if ((rc = dev_alloc(c, &c.dyn.S, fs))) return rc;
    c.dyn_alloc = true;
    return FSL_OK;
}

int ensure_bf(Ctx &c)
{
    if (c.bf_alloc) return FSL_OK;
    const Grid &g = c.g;
    const size_t nx = 5 * (size_t)g.H * g.D, ny = 5 * (size_t)g.L * g.D, nz = 5 * (size_t)g.L * g.H;
    int rc;
    if ((rc = dev_alloc(c, &c.bf.x0, nx))) return rc;
    if ((rc = dev_alloc(c, &c.bf.xL, nx))) return rc;
    if ((rc = dev_alloc(c, &c.bf.y0, ny))) return rc;
    if ((rc = dev_alloc(c, &c.bf.yH, ny))) return rc;
    if ((rc = dev_alloc(c, &c.bf.z0, nz))) return rc;
    if ((rc = dev_alloc(c, &c.bf.zD, nz))) return rc;
    c.bf_alloc = true;
    return FSL_OK;
}

int dev_alloc_f(Ctx &c, float **p, size_t n)
{
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(float));
    if (e != cudaSuccess) {
        *p = nullptr;
        return fail(c, FSL_ERR_NOMEM, "cudaMalloc", e);
    }
    c.bytes += n * sizeof(float);
    e = cudaMemsetAsync(*p, 0, n * sizeof(float), c.stream);
    if (e != cudaSuccess) return fail(c, FSL_ERR_CUDA, "cudaMemsetAsync", e);
    return FSL_OK;
}

int ensure_fp32(Ctx &c)
{
    if (c.fp32_alloc) return FSL_OK;
    const Grid &g = c.g;
    const size_t nx = 5 * (size_t)g.H * g.D, ny = 5 * (size_t)g.L * g.D, nz = 5 * (size_t)g.L * g.H;
    int rc;
    if ((rc = dev_alloc_f(c, &c.bf32.x0, nx))) return rc;
    if ((rc = dev_alloc_f(c, &c.bf32.xL, nx))) return rc;
    if ((rc = dev_alloc_f(c, &c.bf32.y0, ny))) return rc;
    if ((rc = dev_alloc_f(c, &c.bf32.yH, ny))) return rc;
    if ((rc = dev_alloc_f(c, &c.bf32.z0, nz))) return rc;
    if ((rc = dev_alloc_f(c, &c.bf32.zD, nz))) return rc;
    if ((rc = dev_alloc_f(c, &c.mu32, (size_t)g.fstride))) return rc;
    const size_t fs = (size_t)g.fstride;
    if ((rc = dev_alloc_f(c, &c.dyn32.vel, 3 * fs))) return rc;
    if ((rc = dev_alloc_f(c, &c.dyn32.F, 9 * fs))) return rc;
    if ((rc = dev_alloc_f(c, &c.dyn32.A, 6 * fs))) return rc;
    if ((rc = dev_alloc_f(c, &c.dyn32.S, fs))) return rc;
    c.fp32_alloc = true;
    return FSL_OK;
}

double *cur_ptr(Ctx &c) { return c.cur ? c.Up : c.U; }

} // namespace

namespace fsl {
int ensure_dyn_scratch(Ctx &c)
{
    // the dynamic procedure's scratch and, on the FP32 path, the FP32 SGS
    // field it writes (allocated on first use, like the fused step's buffers)
    int rc = ensure_dyn(c);
    if (!rc && c.p.precision == FSL_PREC_FP32) rc = ensure_fp32(c);
    return rc;
}
} // namespace fsl

namespace {

// Disturbance draw of src/layer2.c:152-162 with Random() of src/helpers.c:13-17.
double rnd(double x)
{
    x = 11. * x + 3.14159265358979323846;
    return x - (double)((int)x);
}

void draw(Ctx &c)
{
    const unsigned DEP = (unsigned)c.p.DEP;
    double X = c.X;
    if (c.counter > 0) c.counter--;
    else {
        c.counter = (int)(c.p.Ns_min + c.p.Nst * (X = rnd(X)));
        c.dist.k_min = (unsigned)(DEP * (X = rnd(X)));
        c.dist.k_max = (unsigned)(c.dist.k_min + DEP * (X = rnd(X)));
        if (c.dist.k_max > DEP) c.dist.k_max -= DEP;
        X = rnd(X); c.dist.Ud = c.p.Ua * (1 - X - X);
        X = rnd(X); c.dist.Vd = c.p.Va * (1 - X - X);
        X = rnd(X); c.dist.Wd = c.p.Wa * (1 - X - X);
    }
    c.X = X;
}

int sync_scalars(Ctx &c)
{
    CK(cudaMemcpyAsync(c.hs, c.ds, sizeof(DevScalars), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.dt_host = c.hs->dt;
    c.maxco_host = c.hs->maxCo;
    return FSL_OK;
}

} // namespace

extern "C" {

int fsl_params_default(fsl_params *p)
{
    if (!p) return FSL_ERR_ARG;
    memset(p, 0, sizeof *p);
    p->LEN = 100; p->HIG = 80; p->DEP = 35;
    p->deltaX = 1.6666667; p->deltaY = 1.0; p->deltaZ = 1.5; p->deltaT = 0.0007;
    p->Answer = 0; p->numstep = 3000;
    p->mu_L = 0.253358; p->Pr_L = 0.72; p->Pr_T = 0.8; p->Cs = 0.01;
    p->BL_HIG = 5; p->Ua = 35.; p->Va = 35.; p->Wa = 35.;
    p->Ns_min = 10; p->Nst = 50; p->f_step = 50; p->nStages = 3; p->maxCoNum = 0.1;
    p->setup = FSL_SETUP_SPATIAL; p->cfl_mode = FSL_CFL_STREAMWISE; p->seed_X = 0.317391239817;
    p->precision = FSL_PREC_FP64; p->sgs = FSL_SGS_DYNAMIC; p->recon = FSL_RECON_CHARMINMOD;
    return FSL_OK;
}

static void set_field(fsl_params *p, int i, double v, int from_float)
{
    (void)from_float;
    switch (i) {
    case 0: p->LEN = (int)v; break;
    case 1: p->HIG = (int)v; break;
    case 2: p->DEP = (int)v; break;
    case 3: p->deltaX = v; break;
    case 4: p->deltaY = v; break;
    case 5: p->deltaZ = v; break;
    case 6: p->deltaT = v; break;
    case 7: p->Answer = (int)v; break;
    case 8: p->numstep = (int)v; break;
    case 9: p->mu_L = v; break;
    case 10: p->Pr_L = v; break;
    case 11: p->Pr_T = v; break;
    case 12: p->Cs = v; break;
    case 13: p->BL_HIG = (int)v; break;
    case 14: p->Ua = v; break;
    case 15: p->Va = v; break;
    case 16: p->Wa = v; break;
    case 17: p->Ns_min = (int)v; break;
    case 18: p->Nst = (int)v; break;
    case 19: p->f_step = (int)v; break;
    case 20: p->nStages = (int)v; break;
    case 21: p->maxCoNum = v; break;
    default: break;
    }
}

// src/initialize.c:17-58: 22 lines read with fgets(str, 79, ...), integers
// with atoi and reals with atof (trailing text ignored).
int fsl_params_from_ini(const char *path, fsl_params *p)
{
    if (!path || !p) return FSL_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return FSL_ERR_IO;
    fsl_params q = *p; // option fields are kept as the caller set them
    char str[80];
    int i = 0;
    static const int is_int[22] = {1, 1, 1, 0, 0, 0, 0, 1, 1, 0, 0, 0, 0, 1, 0, 0, 0, 1, 1, 1, 1, 0};
    while (i < 22) {
        if (!fgets(str, 79, f)) {
            fclose(f);
            return FSL_ERR_IO;
        }
        set_field(&q, i, is_int[i] ? (double)atoi(str) : atof(str), 0);
        i++;
    }
    fclose(f);
    *p = q;
    return FSL_OK;
}

// src-par/initialize.c:35-81: 22 native float32 values in ini order,
// assigned to the typed globals by C conversion.
int fsl_params_from_bin(const char *path, fsl_params *p)
{
    if (!path || !p) return FSL_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return FSL_ERR_IO;
    float buf[22];
    size_t n = fread(buf, sizeof(float), 22, f);
    fclose(f);
    if (n != 22) return FSL_ERR_IO;
    fsl_params q = *p; // option fields are kept as the caller set them
    for (int i = 0; i < 22; i++) set_field(&q, i, (double)buf[i], 1);
    *p = q;
    return FSL_OK;
}

int fsl_params_check(const fsl_params *p)
{
    if (!p) return FSL_ERR_ARG;
    if (p->LEN < 2 || p->HIG < 2 || p->DEP < 2) return FSL_ERR_ARG;
    if ((long long)p->LEN * p->HIG * p->DEP > (1LL << 31)) return FSL_ERR_ARG;
    if (!(p->deltaX > 0) || !(p->deltaY > 0) || !(p->deltaZ > 0) || !(p->deltaT > 0)) return FSL_ERR_ARG;
    if (!(p->Pr_L > 0) || !(p->Pr_T > 0) || !(p->maxCoNum > 0)) return FSL_ERR_ARG;
    if (p->nStages < 1 || p->nStages > 3) return FSL_ERR_ARG;
    if (p->setup != FSL_SETUP_SPATIAL && p->setup != FSL_SETUP_TEMPORAL) return FSL_ERR_ARG;
    if (p->cfl_mode != FSL_CFL_STREAMWISE && p->cfl_mode != FSL_CFL_ACOUSTIC) return FSL_ERR_ARG;
    // the disturbance block rows j in [HIG/2, HIG/2+BL_HIG) must exist
    // (src/bounCondOnInterfaces.c:31 writes past the array otherwise)
    if (p->setup == FSL_SETUP_SPATIAL && (p->BL_HIG < 0 || p->HIG / 2 + p->BL_HIG > p->HIG)) return FSL_ERR_ARG;
    if (p->precision != FSL_PREC_FP64 && p->precision != FSL_PREC_FP32) return FSL_ERR_ARG;
    if (p->sgs != FSL_SGS_DYNAMIC && p->sgs != FSL_SGS_LEARNED && p->sgs != FSL_SGS_STATIC && p->sgs != FSL_SGS_NONE)
        return FSL_ERR_ARG;
    if (p->recon != FSL_RECON_CHARMINMOD && p->recon != FSL_RECON_PPM) return FSL_ERR_ARG;
    return FSL_OK;
}

// src/initialize.c:159-187
int fsl_initial_state(const fsl_params *p, double *state)
{
    if (!p || !state || fsl_params_check(p)) return FSL_ERR_ARG;
    const double P = 100000., R = 1.0;
    size_t n = 0;
    for (int i = 1; i <= p->LEN; i++)
        for (int j = 1; j <= p->HIG; j++) {
            const double U = (j <= p->HIG / 2) ? 76.4 : 200;
            const double vals[5] = {R, R * U, 0., 0., P / 0.4 + 0.5 * R * (U * U)};
            for (int v = 0; v < 5; v++)
                for (int k = 0; k < p->DEP; k++) state[n++] = vals[v];
        }
    return FSL_OK;
}

static uint64_t splitmix64(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

int fsl_temporal_state(const fsl_params *p, double Mc, double delta_w0, double amp, unsigned long long seed,
                       double *state, double *dU_out)
{
    if (!p || !state || fsl_params_check(p) || !(delta_w0 > 0) || !(Mc > 0)) return FSL_ERR_ARG;
    const double p0 = 100000., rho0 = 1.0, cp = 717.75 * 1.4, Rg = 287.10;
    const double Tinf = p0 / (Rg * rho0);
    const double cinf = sqrt(1.4 * p0 / rho0);
    const double dU = 2.0 * Mc * cinf;
    const double Ly = p->HIG * p->deltaY;
    uint64_t s = seed;
    size_t n = 0;
    const int D = p->DEP;
    for (int i = 1; i <= p->LEN; i++)
        for (int j = 1; j <= p->HIG; j++) {
            const double y = (j - 0.5) * p->deltaY - 0.5 * Ly;
            const double um = 0.5 * dU * tanh(2.0 * y / delta_w0);
            const double T = Tinf + (0.25 * dU * dU - um * um) / (2.0 * cp);
            const double rho = p0 / (Rg * T);
            double *row = state + n;
            for (int k = 0; k < D; k++) {
                double r3[3];
                for (int q = 0; q < 3; q++)
                    r3[q] = amp * dU * ((double)(splitmix64(&s) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0);
                const double uu = um + r3[0];
                row[k] = rho;
                row[D + k] = rho * uu;
                row[2 * D + k] = rho * r3[1];
                row[3 * D + k] = rho * r3[2];
                row[4 * D + k] = p0 / 0.4 + 0.5 * rho * (uu * uu + r3[1] * r3[1] + r3[2] * r3[2]);
            }
            n += 5 * (size_t)D;
        }
    if (dU_out) *dU_out = dU;
    return FSL_OK;
}

int fsl_init(const fsl_params *p, fsl_ctx **out)
{
    if (!p || !out) return FSL_ERR_ARG;
    *out = nullptr;
    if (fsl_params_check(p)) return FSL_ERR_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FSL_ERR_NODEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return FSL_ERR_NODEVICE;
    if (prop.major != 10) return FSL_ERR_NODEVICE;
    fsl_ctx *h = new (std::nothrow) fsl_ctx();
    if (!h) return FSL_ERR_NOMEM;
    Ctx &c = h->c;
    c.p = *p;
    c.device = dev;
    c.sms = prop.multiProcessorCount > 0 ? prop.multiProcessorCount : 1;
    c.g = make_grid(p->LEN, p->HIG, p->DEP, 8);
    c.co_i0 = 1;
    c.co_i1 = p->LEN;
    // x planes per fused-stage block: 48 measured fastest for the FP32 bulk
    // at 512x256x256 (1.6 % over 32); 32 for FP64
    c.stage_seg = (p->precision == FSL_PREC_FP32) ? 48 : 32;
    // the FP32 bulk's reference-scheme stages run the full-lane persistent
    // tile (rows 0); FP64 and PPM stages the ring tiles (rows 16)
    c.stage_tje = (p->precision == FSL_PREC_FP32) ? 0 : 16;
    // derived constants, src/initialize.c:67-94
    c.k.rdx = 1. / p->deltaX; c.k.rdy = 1. / p->deltaY; c.k.rdz = 1. / p->deltaZ;
    c.k.r4dx = 1. / (4 * p->deltaX); c.k.r4dy = 1. / (4 * p->deltaY); c.k.r4dz = 1. / (4 * p->deltaZ);
    c.k.r2dx = c.k.r4dx + c.k.r4dx; c.k.r2dy = c.k.r4dy + c.k.r4dy; c.k.r2dz = c.k.r4dz + c.k.r4dz;
    c.k.mu_L = p->mu_L;
    c.k.lambda_L = p->mu_L * 717.75 * 1.4 / p->Pr_L;
    c.k.cp_Pr_T = 717.75 * 1.4 / p->Pr_T;
    c.k.DD = pow(p->deltaX * p->deltaY * p->deltaZ, 0.666666666666667);
    c.k.CsDD = p->Cs * c.k.DD;
    c.k.maxCoNum = p->maxCoNum;
    c.k.deltaX = p->deltaX; c.k.deltaY = p->deltaY; c.k.deltaZ = p->deltaZ;
    c.k.setup = p->setup; c.k.BL_HIG = p->BL_HIG; c.k.cfl_mode = p->cfl_mode; c.k.nStages = p->nStages;
    c.X = p->seed_X;
    int rc = FSL_OK;
    if (cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return FSL_ERR_CUDA;
    }
    const size_t fs = (size_t)c.g.fstride;
    if (!rc) rc = dev_alloc(c, &c.U, 5 * fs);
    if (!rc) rc = dev_alloc(c, &c.Up, 5 * fs);
    if (!rc) rc = dev_alloc(c, &c.Uq, 5 * fs);
    if (!rc) rc = dev_alloc(c, &c.mu, fs);
    c.npartials = 148 * 4;
    if (!rc) rc = dev_alloc(c, &c.partials, 4096);
    if (!rc) rc = dev_alloc(c, &c.stage_dev, (size_t)p->LEN * p->HIG * 5 * p->DEP);
    if (!rc) {
        if (cudaMalloc((void **)&c.ds, sizeof(DevScalars)) != cudaSuccess) rc = FSL_ERR_NOMEM;
        else if (cudaMallocHost((void **)&c.hs, sizeof(DevScalars)) != cudaSuccess) rc = FSL_ERR_NOMEM;
    }
    if (!rc) {
        memset(c.hs, 0, sizeof(DevScalars));
        c.hs->dt = p->deltaT;
        c.hs->dtx = p->deltaT / p->deltaX; c.hs->dty = p->deltaT / p->deltaY; c.hs->dtz = p->deltaT / p->deltaZ;
        if (cudaMemcpyAsync(c.ds, c.hs, sizeof(DevScalars), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
            cudaStreamSynchronize(c.stream) != cudaSuccess)
            rc = FSL_ERR_CUDA;
        c.dt_host = p->deltaT;
    }
    if (rc) {
        fsl_destroy(h);
        return rc;
    }
    *out = h;
    return FSL_OK;
}

int fsl_destroy(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(c.U); cudaFree(c.Up); cudaFree(c.Uq); cudaFree(c.mu);
    cudaFree(c.partials); cudaFree(c.stage_dev); cudaFree(c.ds); cudaFree(c.favre);
    if (c.xfer_alloc) {
        if (c.up) cudaStreamSynchronize(c.up);
        if (c.down) cudaStreamSynchronize(c.down);
        cudaFree(c.xin); cudaFree(c.xout);
        cudaEvent_t *ev[4] = {&c.ev_in_ready, &c.ev_in_free, &c.ev_out_ready, &c.ev_out_free};
        for (cudaEvent_t *e : ev)
            if (*e) cudaEventDestroy(*e);
        if (c.up) cudaStreamDestroy(c.up);
        if (c.down) cudaStreamDestroy(c.down);
    }
    if (c.hs) cudaFreeHost(c.hs);
    if (c.faces_alloc)
        for (int s = 0; s < 2; s++)
            for (int v = 0; v < 5; v++) { cudaFree(c.f.x[s][v]); cudaFree(c.f.y[s][v]); cudaFree(c.f.z[s][v]); }
    if (c.dyn_alloc) {
        cudaFree(c.dyn.vel); cudaFree(c.dyn.F); cudaFree(c.dyn.A); cudaFree(c.dyn.S);
    }
    if (c.bf_alloc) {
        cudaFree(c.bf.x0); cudaFree(c.bf.xL); cudaFree(c.bf.y0);
        cudaFree(c.bf.yH); cudaFree(c.bf.z0); cudaFree(c.bf.zD);
    }
    closure_free(c);
    if (c.fp32_alloc) {
        cudaFree(c.bf32.x0); cudaFree(c.bf32.xL); cudaFree(c.bf32.y0);
        cudaFree(c.bf32.yH); cudaFree(c.bf32.z0); cudaFree(c.bf32.zD); cudaFree(c.mu32);
        cudaFree(c.dyn32.vel); cudaFree(c.dyn32.F); cudaFree(c.dyn32.A); cudaFree(c.dyn32.S);
    }
    for (auto &r : c.recs) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : c.evpool) cudaEventDestroy(e);
    if (c.open_ev) cudaEventDestroy(c.open_ev);
    if (c.stream) cudaStreamDestroy(c.stream);
    delete h;
    return FSL_OK;
}

const char *fsl_last_error(const fsl_ctx *h)
{
    if (!h) return kNoCtx;
    return h->c.err.c_str();
}

int fsl_sync(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = sync_scalars(c);
    if (rc) return rc;
    if (c.hs->status) return fail(c, FSL_ERR_NONFINITE, "non-finite or non-positive Courant maximum or density");
    return FSL_OK;
}

int fsl_get_info(fsl_ctx *h, fsl_info *info)
{
    if (!h || !info) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = sync_scalars(c);
    if (rc) return rc;
    memset(info, 0, sizeof *info);
    info->deltaT = c.hs->dt; info->deltaT_X = c.hs->dtx; info->deltaT_Y = c.hs->dty; info->deltaT_Z = c.hs->dtz;
    info->maxCo = c.hs->maxCo;
    info->X = c.X; info->Ud = c.dist.Ud; info->Vd = c.dist.Vd; info->Wd = c.dist.Wd;
    info->k_min = c.dist.k_min; info->k_max = c.dist.k_max;
    info->step = c.step; info->counter = c.counter; info->cur = c.cur;
    info->DD = c.k.DD; info->lambda_L = c.k.lambda_L; info->cp_Pr_T = c.k.cp_Pr_T;
    info->device_bytes = c.bytes;
    return FSL_OK;
}

int fsl_upload_state(fsl_ctx *h, const double *state)
{
    ApiRange range_("fsl_upload_state");
    if (!h || !state) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    c.co_valid = false;
    c.stage_next = 0; // a step in progress is abandoned
    CK(cudaMemcpyAsync(c.stage_dev, state, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    launch_state_scatter(c, c.U, c.stage_dev, 1, c.p.LEN);
    CKL();
    // a new state: the flags of the one it replaces are cleared
    CK(cudaMemsetAsync(&c.ds->status, 0, sizeof c.ds->status, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.cur = 0;
    return FSL_OK;
}

int fsl_download_state(fsl_ctx *h, double *state)
{
    ApiRange range_("fsl_download_state");
    if (!h || !state) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    launch_state_gather(c, c.U, c.stage_dev, 1, c.p.LEN);
    CKL();
    CK(cudaMemcpyAsync(state, c.stage_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

// ---- x-slabs ----------------------------------------------------------------
// A decomposed domain is a set of contexts, one per slab of x-planes (one per
// GPU), each holding its own planes plus overlap planes copied from its
// neighbours once per step.  These calls move planes in and out of U^n and
// make the Courant maximum (src/helpers.c:23-52) a maximum over the owned
// planes, to be combined across slabs before the next step.

static bool planes_ok(const Ctx &c, int i0, int n)
{
    return i0 >= 1 && n >= 0 && i0 + n - 1 <= c.p.LEN;
}

// the buffer holding the current stage state: U^n between steps, the output
// of stage 1 or 2 while fsl_step_stage is in the middle of a step
static double *stage_state(Ctx &c)
{
    return c.stage_next == 2 ? c.Up : c.stage_next == 3 ? c.Uq : c.U;
}

// gather planes i0.. of the current stage state into buf, queued on the
// context's stream (the one scratch buffer is reused in stream order)
static int get_planes_q(fsl_ctx *h, int i0, int n, double *buf)
{
    ApiRange range_("fsl_get_planes");
    if (!h || !buf || !planes_ok(h->c, i0, n)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_get_planes: the current-stage buffer is not U^n");
    const size_t bytes = (size_t)n * c.p.HIG * 5 * c.p.DEP * sizeof(double);
    launch_state_gather(c, stage_state(c), c.stage_dev, i0, n);
    CKL();
    if (bytes) CK(cudaMemcpyAsync(buf, c.stage_dev, bytes, cudaMemcpyDefault, c.stream));
    return FSL_OK;
}

static int set_planes_q(fsl_ctx *h, int i0, int n, const double *buf)
{
    ApiRange range_("fsl_set_planes");
    if (!h || !buf || !planes_ok(h->c, i0, n)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_set_planes: the current-stage buffer is not U^n");
    const size_t bytes = (size_t)n * c.p.HIG * 5 * c.p.DEP * sizeof(double);
    // planes outside the Courant range leave the owned maximum as it is
    if (c.stage_next == 0 && n > 0 && i0 <= c.co_i1 && i0 + n - 1 >= c.co_i0) c.co_valid = false;
    if (bytes) CK(cudaMemcpyAsync(c.stage_dev, buf, bytes, cudaMemcpyDefault, c.stream));
    launch_state_scatter(c, stage_state(c), c.stage_dev, i0, n);
    CKL();
    return FSL_OK;
}

int fsl_get_planes(fsl_ctx *h, int i0, int n, double *buf)
{
    const int rc = get_planes_q(h, i0, n, buf);
    if (rc) return rc;
    Ctx &c = h->c;
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_set_planes(fsl_ctx *h, int i0, int n, const double *buf)
{
    const int rc = set_planes_q(h, i0, n, buf);
    if (rc) return rc;
    Ctx &c = h->c;
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_get_planes_async(fsl_ctx *h, int i0, int n, double *buf) { return get_planes_q(h, i0, n, buf); }

int fsl_set_planes_async(fsl_ctx *h, int i0, int n, const double *buf) { return set_planes_q(h, i0, n, buf); }

int fsl_set_courant_range(fsl_ctx *h, int i0, int i1)
{
    if (!h || i0 < 1 || i1 < i0 || i1 > h->c.p.LEN) return FSL_ERR_ARG;
    Ctx &c = h->c;
    c.co_i0 = i0;
    c.co_i1 = i1;
    c.co_valid = false;
    return FSL_OK;
}

int fsl_courant_prepare(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_courant_prepare: the current-stage buffer is not U^n");
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "a step is in progress (fsl_step_stage)");
    if (!c.co_valid) {
        launch_courant_to_bits(c);
        CKL();
        c.co_valid = true;
    }
    return FSL_OK;
}

unsigned long long *fsl_courant_bits(fsl_ctx *h)
{
    return h ? &h->c.ds->co_bits : nullptr;
}

int fsl_get_courant_max(fsl_ctx *h, double *maxCo)
{
    if (!h || !maxCo) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (!c.co_valid) return fail(c, FSL_ERR_ARG, "fsl_get_courant_max: no maximum for the current state");
    unsigned long long b = 0;
    CK(cudaMemcpyAsync(&b, &c.ds->co_bits, sizeof b, cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    memcpy(maxCo, &b, sizeof b);
    return FSL_OK;
}

int fsl_set_courant_max(fsl_ctx *h, double maxCo)
{
    if (!h || !(maxCo >= 0.0)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    // the final stage of a step in progress accumulates into the same scalar
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "a step is in progress (fsl_step_stage)");
    unsigned long long b;
    memcpy(&b, &maxCo, sizeof b);
    CK(cudaMemcpyAsync(&c.ds->co_bits, &b, sizeof b, cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.co_valid = true;
    return FSL_OK;
}

// ---- asynchronous state transfer ----------------------------------------------
static int ensure_xfer(Ctx &c)
{
    if (c.xfer_alloc) return FSL_OK;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    if (cudaMalloc((void **)&c.xin, n * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void **)&c.xout, n * sizeof(double)) != cudaSuccess) {
        cudaFree(c.xin); cudaFree(c.xout);
        c.xin = c.xout = nullptr;
        return fail(c, FSL_ERR_NOMEM, "asynchronous transfer buffers");
    }
    c.xfer_alloc = true;
    c.bytes += 2 * n * sizeof(double);
    CK(cudaStreamCreateWithFlags(&c.up, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c.down, cudaStreamNonBlocking));
    cudaEvent_t *ev[4] = {&c.ev_in_ready, &c.ev_in_free, &c.ev_out_ready, &c.ev_out_free};
    for (cudaEvent_t *e : ev) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    // both staging buffers start free
    CK(cudaEventRecord(c.ev_in_free, c.stream));
    CK(cudaEventRecord(c.ev_out_free, c.stream));
    return FSL_OK;
}

// The H2D copy runs on its own stream as soon as the previous scatter has
// left the staging buffer, so it overlaps the work queued before it; the
// scatter into U^n is queued on the context's stream behind that work.
int fsl_upload_state_async(fsl_ctx *h, const double *state)
{
    ApiRange range_("fsl_upload_state_async");
    if (!h || !state) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_xfer(c);
    if (rc) return rc;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    c.co_valid = false;
    c.stage_next = 0; // a step in progress is abandoned
    CK(cudaStreamWaitEvent(c.up, c.ev_in_free, 0));
    CK(cudaMemcpyAsync(c.xin, state, n * sizeof(double), cudaMemcpyHostToDevice, c.up));
    CK(cudaEventRecord(c.ev_in_ready, c.up));
    CK(cudaStreamWaitEvent(c.stream, c.ev_in_ready, 0));
    launch_state_scatter(c, c.U, c.xin, 1, c.p.LEN);
    CKL();
    CK(cudaEventRecord(c.ev_in_free, c.stream));
    c.cur = 0;
    return FSL_OK;
}

// The gather out of U^n is queued on the context's stream (once the previous
// D2H copy has left the staging buffer); the D2H copy runs on its own stream
// and overlaps the work queued after it.
int fsl_download_state_async(fsl_ctx *h, double *state)
{
    ApiRange range_("fsl_download_state_async");
    if (!h || !state) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_xfer(c);
    if (rc) return rc;
    if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_download_state_async: the current-stage buffer is not U^n");
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    CK(cudaStreamWaitEvent(c.stream, c.ev_out_free, 0));
    launch_state_gather(c, c.U, c.xout, 1, c.p.LEN);
    CKL();
    CK(cudaEventRecord(c.ev_out_ready, c.stream));
    CK(cudaStreamWaitEvent(c.down, c.ev_out_ready, 0));
    CK(cudaMemcpyAsync(state, c.xout, n * sizeof(double), cudaMemcpyDeviceToHost, c.down));
    CK(cudaEventRecord(c.ev_out_free, c.down));
    return FSL_OK;
}

int fsl_transfer_wait(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.xfer_alloc) {
        CK(cudaStreamSynchronize(c.up));
        CK(cudaStreamSynchronize(c.down));
    }
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_set_time(fsl_ctx *h, unsigned step, double deltaT)
{
    if (!h || !(deltaT > 0)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = sync_scalars(c);
    if (rc) return rc;
    c.co_valid = false;
    c.step = step;
    c.hs->dt = deltaT;
    c.hs->dtx = deltaT / c.p.deltaX; c.hs->dty = deltaT / c.p.deltaY; c.hs->dtz = deltaT / c.p.deltaZ;
    CK(cudaMemcpyAsync(c.ds, c.hs, sizeof(DevScalars), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    c.dt_host = deltaT;
    return FSL_OK;
}

int fsl_check_courant(fsl_ctx *h, double *maxCo, double *dt)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "a step is in progress (fsl_step_stage)");
    c.co_valid = false;
    launch_courant(c);
    CKL();
    int rc = sync_scalars(c);
    if (rc) return rc;
    if (maxCo) *maxCo = c.hs->maxCo;
    if (dt) *dt = c.hs->dt;
    if (c.hs->status) return fail(c, FSL_ERR_NONFINITE, "non-finite or non-positive Courant maximum or density");
    return FSL_OK;
}

int fsl_draw_disturbance(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    draw(h->c);
    return FSL_OK;
}

int fsl_set_disturbance(fsl_ctx *h, unsigned k_min, unsigned k_max, double Ud, double Vd, double Wd)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    c.dist.k_min = k_min; c.dist.k_max = k_max; c.dist.Ud = Ud; c.dist.Vd = Vd; c.dist.Wd = Wd;
    return FSL_OK;
}

int fsl_ghost_bc(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_ghost_bc: a step is in progress (fsl_step_stage)");
    launch_ghost(c, cur_ptr(c));
    CKL();
    return FSL_OK;
}

int fsl_reconstruct(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_reconstruct: a step is in progress (fsl_step_stage)");
    int rc = ensure_faces(c);
    if (rc) return rc;
    launch_recon(c, cur_ptr(c));
    CKL();
    return FSL_OK;
}

int fsl_interface_bc(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_interface_bc: a step is in progress (fsl_step_stage)");
    int rc = ensure_faces(c);
    if (rc) return rc;
    launch_ifbc(c, c.dist);
    CKL();
    return FSL_OK;
}

int fsl_dynamic_smagorinsky(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_dynamic_smagorinsky: a step is in progress (fsl_step_stage)");
    int rc = ensure_dyn(c);
    if (rc) return rc;
    launch_dynsmag(c, c.U);
    CKL();
    return FSL_OK;
}

int fsl_fluxes(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_fluxes: a step is in progress (fsl_step_stage)");
    int rc = ensure_faces(c);
    if (rc) return rc;
    launch_fluxes(c, cur_ptr(c));
    CKL();
    return FSL_OK;
}

int fsl_evolution(fsl_ctx *h, int stage)
{
    if (!h || stage < 1) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "fsl_evolution: a step is in progress (fsl_step_stage)");
    int rc = ensure_faces(c);
    if (rc) return rc;
    c.co_valid = false;
    launch_evolution(c, c.p.nStages, stage);
    CKL();
    // pointer swap of src/evolution.c:71,113,155 (and :188,228 for RK2)
    c.cur = (stage == 1 || stage == 2) ? 1 : 0;
    return FSL_OK;
}

// The FP32 bulk's full-lane stages on the temporal setup form the boundary
// faces' outer states from the state itself and write the ghost cells of
// their output: no boundary pass runs, and no ghost pass between stages.
static bool wide_temporal(const Ctx &c)
{
    return c.p.precision == FSL_PREC_FP32 && c.p.recon == FSL_RECON_CHARMINMOD && c.stage_tje == 0 &&
           c.p.setup == FSL_SETUP_TEMPORAL;
}

// The SGS viscosity of one step, on U^n with its ghost layer filled: the
// dynamic procedure, the learned closure (judged by the dynamic procedure),
// nothing for the static model (the stage kernels form it per face), or a
// zero field.
static int step_sgs(Ctx &c)
{
    const bool fp32 = c.p.precision == FSL_PREC_FP32;
    switch (c.p.sgs) {
    case FSL_SGS_LEARNED: return closure_step_sgs(c);
    case FSL_SGS_STATIC: return FSL_OK;
    case FSL_SGS_NONE:
        if (fp32) CK(cudaMemsetAsync(c.mu32, 0, (size_t)c.g.fstride * sizeof(float), c.stream));
        else CK(cudaMemsetAsync(c.mu, 0, (size_t)c.g.fstride * sizeof(double), c.stream));
        return FSL_OK;
    default:
        if (fp32) launch_dynsmag32(c, c.U);
        else launch_dynsmag(c, c.U);
        return FSL_OK;
    }
}

} // extern "C"

namespace fsl {
// The part of an FP32-bulk fused step before its stages, for the persistent
// multi-domain stage launch (which runs the three stages, with the ghost
// layers and boundary faces between them): the same launches fsl_step makes
// before its first stage.
int step_prelude32(Ctx &c)
{
    int rc;
    if ((rc = ensure_dyn(c)) || (rc = ensure_bf(c)) || (rc = ensure_fp32(c))) return rc;
    if (c.co_valid) launch_courant_apply(c);
    else launch_courant(c);
    c.step++;
    draw(c);
    launch_ghost(c, c.U);
    if (!wide_temporal(c)) launch_bface32(c, c.U, c.dist);
    return step_sgs(c);
}
} // namespace fsl

extern "C" {

// An x-slab (Courant range narrower than the domain) steps one step at a
// time, from a Courant maximum combined across the slabs; a learned closure
// would judge on the slab alone.
static int slab_check(Ctx &c, int nsteps)
{
    if (c.stage_next != 0) return fail(c, FSL_ERR_ARG, "a step is in progress (fsl_step_stage)");
    if (c.co_i0 == 1 && c.co_i1 == c.p.LEN) return FSL_OK;
    if (nsteps > 1) return fail(c, FSL_ERR_ARG, "x-slab: one step per call (overlap exchange between steps)");
    if (nsteps == 1 && !c.co_valid)
        return fail(c, FSL_ERR_ARG, "x-slab: no combined Courant maximum (fsl_courant_prepare / fsl_set_courant_max)");
    if (c.p.sgs == FSL_SGS_LEARNED && c.judge_every > 0)
        return fail(c, FSL_ERR_UNSUPPORTED, "x-slab: closure judgements would differ between slabs");
    return FSL_OK;
}

static bool is_slab(const Ctx &c)
{
    return c.co_i0 != 1 || c.co_i1 != c.p.LEN;
}

int fsl_step_phased(fsl_ctx *h, int nsteps)
{
    ApiRange range_("fsl_step_phased");
    if (!h || nsteps < 0) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc;
    if ((rc = slab_check(c, nsteps))) return rc;
    for (int n = 0; n < nsteps; n++) {
        if (c.co_valid) launch_courant_apply(c);
        else launch_courant(c);
        CKL();
        c.step++;
        draw(c);
        for (int s = 1; s <= c.p.nStages; s++) {
            if ((rc = ensure_faces(c))) return rc;
            if ((rc = ensure_dyn(c))) return rc;
            double *cur = cur_ptr(c);
            launch_ghost(c, cur);
            launch_recon(c, cur);
            launch_ifbc(c, c.dist);
            if (s == 1) {
                if (c.p.sgs == FSL_SGS_NONE) CK(cudaMemsetAsync(c.mu, 0, (size_t)c.g.fstride * sizeof(double), c.stream));
                else if (c.p.sgs != FSL_SGS_STATIC) launch_dynsmag(c, c.U);
            }
            launch_fluxes(c, cur);
            launch_evolution(c, c.p.nStages, s);
            c.cur = (s == 1 || s == 2) ? 1 : 0;
            CKL();
        }
        c.co_valid = false;
        if (is_slab(c)) {
            // the owned maximum of the new state, to be combined across slabs
            launch_courant_to_bits(c);
            CKL();
            c.co_valid = true;
        }
    }
    return FSL_OK;
}

// Fused path: per stage a ghost fill, the boundary outer states and one
// fused stage kernel; stages ping-pong U^n -> Up -> Uq -> U^n.
int fsl_step(fsl_ctx *h, int nsteps)
{
    ApiRange range_("fsl_step");
    if (!h || nsteps < 0) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.p.nStages != 3) {
        // the RK2 chain runs on the per-phase kernels (FP64)
        if (c.p.precision != FSL_PREC_FP64) return fail(c, FSL_ERR_UNSUPPORTED, "FP32 bulk needs nStages = 3");
        return fsl_step_phased(h, nsteps);
    }
    int rc;
    if ((rc = slab_check(c, nsteps))) return rc;
    if ((rc = ensure_dyn(c))) return rc;
    if ((rc = ensure_bf(c))) return rc;
    if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_step: the current-stage buffer is not U^n");
    if (c.p.precision == FSL_PREC_FP32) {
        if ((rc = ensure_fp32(c))) return rc;
        const bool wt = wide_temporal(c);
        // the learned closure's feature velocities: the last stage of a step
        // writes those of U^{n+1}, so only the first step of a call (whose
        // U^n the caller may have written) runs the velocity pass
        float *vel = (wt && c.p.sgs == FSL_SGS_LEARNED && c.cl_alloc) ? c.cl_vel : nullptr;
        for (int n = 0; n < nsteps; n++) {
            if (c.co_valid) launch_courant_apply(c);
            else launch_courant(c);
            c.step++;
            draw(c);
            // U^n's ghost layer: the previous step's last stage wrote it,
            // unless that step ran before this call
            if (!wt || n == 0) launch_ghost(c, c.U);
            if (!wt) launch_bface32(c, c.U, c.dist);
            c.vel_fresh = vel && n > 0;
            rc = step_sgs(c);
            c.vel_fresh = false;
            if (rc) return rc;
            if (launch_stage32(c, 1, c.U, c.U, c.Up)) return fail(c, FSL_ERR_CUDA, "FP32 stage kernel");
            if (!wt) {
                launch_ghost(c, c.Up);
                launch_bface32(c, c.Up, c.dist);
            }
            launch_stage32(c, 2, c.Up, c.U, c.Uq);
            if (!wt) {
                launch_ghost(c, c.Uq);
                launch_bface32(c, c.Uq, c.dist);
            }
            launch_stage32(c, 3, c.Uq, c.U, c.U, true, vel);
            c.co_valid = true;
            CKL();
        }
        return FSL_OK;
    }
    for (int n = 0; n < nsteps; n++) {
        if (c.co_valid) launch_courant_apply(c);
        else launch_courant(c);
        c.step++;
        draw(c);
        launch_ghost(c, c.U);
        launch_bface(c, c.U, c.dist);
        if ((rc = step_sgs(c))) return rc;
        if (launch_stage(c, 1, c.U, c.U, c.Up)) return fail(c, FSL_ERR_CUDA, "stage kernel attribute");
        launch_ghost(c, c.Up);
        launch_bface(c, c.Up, c.dist);
        launch_stage(c, 2, c.Up, c.U, c.Uq);
        launch_ghost(c, c.Uq);
        launch_bface(c, c.Uq, c.dist);
        launch_stage(c, 3, c.Uq, c.U, c.U, true);
        c.co_valid = true;
        CKL();
    }
    return FSL_OK;
}

// One RK stage of the fused step, the three in turn: the first begins the
// step (Courant rescale, disturbance draw, SGS viscosity, stage 1), the third
// completes it.  The same launches as fsl_step, so an x-slab can refresh its
// overlap planes between stages.
int fsl_step_stage(fsl_ctx *h)
{
    ApiRange range_("fsl_step_stage");
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (c.p.nStages != 3) return fail(c, FSL_ERR_UNSUPPORTED, "fsl_step_stage: nStages = 3 only");
    const bool fp32 = c.p.precision == FSL_PREC_FP32;
    int rc;
    if (c.stage_next == 0) {
        if ((rc = slab_check(c, 1))) return rc;
        if ((rc = ensure_dyn(c))) return rc;
        if ((rc = ensure_bf(c))) return rc;
        if (fp32 && (rc = ensure_fp32(c))) return rc;
        if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_step_stage: the current-stage buffer is not U^n");
        if (c.co_valid) launch_courant_apply(c);
        else launch_courant(c);
        c.step++;
        draw(c);
        launch_ghost(c, c.U);
        if (fp32) launch_bface32(c, c.U, c.dist);
        else launch_bface(c, c.U, c.dist);
        if ((rc = step_sgs(c))) return rc;
        const int e = fp32 ? launch_stage32(c, 1, c.U, c.U, c.Up) : launch_stage(c, 1, c.U, c.U, c.Up);
        if (e) return fail(c, FSL_ERR_CUDA, "stage kernel");
        c.stage_next = 2;
    } else if (c.stage_next == 2) {
        if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_step_stage: the current-stage buffer is not U^n");
        launch_ghost(c, c.Up);
        if (fp32) {
            launch_bface32(c, c.Up, c.dist);
            launch_stage32(c, 2, c.Up, c.U, c.Uq);
        } else {
            launch_bface(c, c.Up, c.dist);
            launch_stage(c, 2, c.Up, c.U, c.Uq);
        }
        c.stage_next = 3;
    } else {
        if (c.cur != 0) return fail(c, FSL_ERR_ARG, "fsl_step_stage: the current-stage buffer is not U^n");
        launch_ghost(c, c.Uq);
        if (fp32) {
            launch_bface32(c, c.Uq, c.dist);
            launch_stage32(c, 3, c.Uq, c.U, c.U, true);
        } else {
            launch_bface(c, c.Uq, c.dist);
            launch_stage(c, 3, c.Uq, c.U, c.U, true);
        }
        c.co_valid = true;
        c.stage_next = 0;
    }
    CKL();
    return FSL_OK;
}

int fsl_debug_bounds(fsl_bounds_report *out, int clear)
{
    if (!out) return FSL_ERR_ARG;
    *out = fsl_bounds_report{};
#if FSL_BOUNDS_CHECK
    if (cudaDeviceSynchronize() != cudaSuccess) return FSL_ERR_CUDA;
    int (*const readers[6])(chk::Record *, bool) = {chk_read_fused, chk_read_fused32, chk_read_mlp, chk_read_phase,
                                                    chk_read_dyn32, chk_read_io};
    for (int u = 0; u < 6; u++) {
        chk::Record r{};
        if (readers[u](&r, clear != 0) != 0) return FSL_ERR_CUDA;
        if (r.hits && !out->hits) {
            out->unit = u + 1;
            out->line = r.line;
            out->index = r.index;
            out->extent = r.extent;
        }
        out->hits += r.hits;
    }
    return FSL_OK;
#else
    (void)clear;
    return FSL_ERR_UNSUPPORTED;
#endif
}

int fsl_tune(fsl_ctx *h, int key, int value)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    switch (key) {
    case FSL_TUNE_STAGE_ROWS:
        if (value != 0 && value != 8 && value != 12 && value != 16) return FSL_ERR_ARG;
        c.stage_tje = value;
        return FSL_OK;
    case FSL_TUNE_STAGE_SEG:
        if (value < 1 || value > 1 << 20) return FSL_ERR_ARG;
        c.stage_seg = value;
        return FSL_OK;
    case FSL_TUNE_CLOSURE_POLY:
        if (value < 0 || value > 6 || value == 1) return FSL_ERR_ARG;
        c.infer_poly = value;
        return FSL_OK;
    default:
        return FSL_ERR_ARG;
    }
}

int fsl_get_cells(fsl_ctx *h, int which, int var, double *out)
{
    if (!h || !out || var < 0 || var > 4 || which < 0 || which > 3) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const Grid &g = c.g;
    const double *base = which == 0 ? c.U : which == 1 ? c.Up : which == 2 ? cur_ptr(c) : c.mu;
    if (which == 3) var = 0;
    base += var * g.fstride + g.off;
    CK(cudaMemcpy2DAsync(out, (g.D + 2) * sizeof(double), base, g.pk * sizeof(double), (g.D + 2) * sizeof(double),
                         (size_t)(g.L + 2) * (g.H + 2), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_set_cells(fsl_ctx *h, int which, int var, const double *in)
{
    if (!h || !in || var < 0 || var > 4 || which < 0 || which > 3) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const Grid &g = c.g;
    double *base = which == 0 ? c.U : which == 1 ? c.Up : which == 2 ? cur_ptr(c) : c.mu;
    if (which == 3) var = 0;
    base += var * g.fstride + g.off;
    c.co_valid = false;
    CK(cudaMemcpy2DAsync(base, g.pk * sizeof(double), in, (g.D + 2) * sizeof(double), (g.D + 2) * sizeof(double),
                         (size_t)(g.L + 2) * (g.H + 2), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_get_faces(fsl_ctx *h, int dir, int side, int var, double *out)
{
    if (!h || !out || dir < 0 || dir > 2 || side < 0 || side > 1 || var < 0 || var > 4) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_faces(c);
    if (rc) return rc;
    const double *p = dir == 0 ? c.f.x[side][var] : dir == 1 ? c.f.y[side][var] : c.f.z[side][var];
    CK(cudaMemcpyAsync(out, p, face_count(c.g, dir) * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_set_faces(fsl_ctx *h, int dir, int side, int var, const double *in)
{
    if (!h || !in || dir < 0 || dir > 2 || side < 0 || side > 1 || var < 0 || var > 4) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_faces(c);
    if (rc) return rc;
    double *p = dir == 0 ? c.f.x[side][var] : dir == 1 ? c.f.y[side][var] : c.f.z[side][var];
    CK(cudaMemcpyAsync(p, in, face_count(c.g, dir) * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_set_cur(fsl_ctx *h, int which)
{
    if (!h || which < 0 || which > 1) return FSL_ERR_ARG;
    h->c.co_valid = false;
    h->c.cur = which;
    return FSL_OK;
}

int fsl_profile(fsl_ctx *h, int on)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    CK(cudaStreamSynchronize(c.stream));
    for (auto &r : c.recs) { c.evpool.push_back(r.a); c.evpool.push_back(r.b); }
    c.recs.clear();
    for (int k = 0; k < FSL_K_COUNT; k++) { c.kms[k] = 0; c.klaunch[k] = 0; }
    c.prof = on != 0;
    return FSL_OK;
}

int fsl_profile_read(fsl_ctx *h, fsl_ktimes *out)
{
    if (!h || !out) return FSL_ERR_ARG;
    Ctx &c = h->c;
    CK(cudaStreamSynchronize(c.stream));
    for (auto &r : c.recs) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, r.a, r.b));
        c.kms[r.cls] += ms;
        c.evpool.push_back(r.a);
        c.evpool.push_back(r.b);
    }
    c.recs.clear();
    for (int k = 0; k < FSL_K_COUNT; k++) { out->ms[k] = c.kms[k]; out->launches[k] = c.klaunch[k]; }
    return FSL_OK;
}

void *fsl_stream(fsl_ctx *h) { return h ? (void *)h->c.stream : nullptr; }

int fsl_sums(fsl_ctx *h, double sums[5])
{
    if (!h || !sums) return FSL_ERR_ARG;
    Ctx &c = h->c;
    double *d = c.partials + 4000;
    launch_sums(c, c.U, c.co_i0, c.co_i1 - c.co_i0 + 1, d);
    CKL();
    CK(cudaMemcpyAsync(sums, d, 5 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

int fsl_plane_sums(fsl_ctx *h, double *rows)
{
    if (!h || !rows) return FSL_ERR_ARG;
    Ctx &c = h->c;
    double *d = c.stage_dev; // scratch: 8*HIG <= LEN*HIG*5*DEP
    launch_plane_sums(c, c.U, c.co_i0, c.co_i1 - c.co_i0 + 1, d);
    CKL();
    CK(cudaMemcpyAsync(rows, d, 8 * (size_t)c.p.HIG * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return FSL_OK;
}

} // extern "C"
