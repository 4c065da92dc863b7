// fsl_closure.cu -- host side of the learned subgrid closure: weights, the
// per-step SGS selection (MLP, or the dynamic procedure as judge/fallback),
// sample harvest and the Adam training driver.  The tensor-core kernels are
// in fsl_mlp.cu.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "fsl_internal.h"

using namespace fsl;


struct fsl_trainer {
    long long cap = 0, n = 0;
    float *X = nullptr, *Y = nullptr;      // samples
    float *P = nullptr, *M = nullptr, *V = nullptr;
    float *Gpart = nullptr, *Gout = nullptr, *lossp = nullptr;
    int *err = nullptr;
    int maxblk = 148;
    long long adam_t = 0;
    bool shuffled = false;
    int loss_mode = 1;      // 0: MSE of Cs^2, 1: weighted by (rho |S| t_ref)^2 (MSE of mu_SGS)
    float inv_wmean = 0.f;  // 1 / mean weight of the current samples (0 = not computed)
    unsigned long long seed = 0;
    cudaStream_t st = nullptr;
};

namespace {

uint64_t splitmix(uint64_t &s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

double unif(uint64_t &s) { return (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

// He-uniform weights, zero biases; the padded inputs 8..15 of W1 are zero.
void init_params(std::vector<float> &p, uint64_t seed)
{
    p.assign(kNParams, 0.f);
    uint64_t s = seed;
    const double a1 = std::sqrt(6.0 / 8.0), a = std::sqrt(6.0 / 64.0);
    for (int o = 0; o < 64; o++)
        for (int i = 0; i < 8; i++) p[kOffW1 + o * 16 + i] = (float)(a1 * (2 * unif(s) - 1));
    for (int e = 0; e < 64 * 64; e++) p[kOffW2 + e] = (float)(a * (2 * unif(s) - 1));
    for (int e = 0; e < 64 * 64; e++) p[kOffW3 + e] = (float)(a * (2 * unif(s) - 1));
    for (int e = 0; e < 64; e++) p[kOffW4 + e] = (float)(0.1 * a * (2 * unif(s) - 1));
}

int ensure_closure(Ctx &c)
{
    if (c.cl_alloc) return FSL_OK;
    const size_t fs = (size_t)c.g.fstride;
    if (cudaMalloc((void **)&c.cl_params, kNParams * sizeof(float)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMalloc((void **)&c.cd32, fs * sizeof(float)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMalloc((void **)&c.cs2_32, fs * sizeof(float)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMalloc((void **)&c.cl_err, sizeof(int)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMalloc((void **)&c.cl_vel, 3 * fs * sizeof(float)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMalloc((void **)&c.judge_rows, 8 * (size_t)c.g.H * sizeof(double)) != cudaSuccess) return FSL_ERR_NOMEM;
    if (c.p.precision == FSL_PREC_FP32) {
        if (cudaMalloc((void **)&c.mu32_alt, fs * sizeof(float)) != cudaSuccess) return FSL_ERR_NOMEM;
        cudaMemsetAsync(c.mu32_alt, 0, fs * sizeof(float), c.stream);
    } else {
        if (cudaMalloc((void **)&c.mu_alt, fs * sizeof(double)) != cudaSuccess) return FSL_ERR_NOMEM;
        cudaMemsetAsync(c.mu_alt, 0, fs * sizeof(double), c.stream);
    }
    cudaMemsetAsync(c.cd32, 0, fs * sizeof(float), c.stream);
    cudaMemsetAsync(c.cs2_32, 0, fs * sizeof(float), c.stream);
    cudaMemsetAsync(c.cl_err, 0, sizeof(int), c.stream);
    cudaMemsetAsync(c.cl_vel, 0, 3 * fs * sizeof(float), c.stream);
    c.bytes += fs * (sizeof(float) * 6 + sizeof(double)) + kNParams * sizeof(float);
    c.cl_alloc = true;
    return FSL_OK;
}

int set_scales(Ctx &c, double t_ref, double len_ref)
{
    if (!(t_ref > 0) || !(len_ref > 0)) return FSL_ERR_ARG;
    const double vol = c.p.deltaX * c.p.deltaY * c.p.deltaZ;
    c.cls.t_ref = (float)t_ref;
    c.cls.delta_ratio = (float)(std::cbrt(vol) / len_ref);
    c.cls.r2dx = (float)c.k.r2dx;
    c.cls.r2dy = (float)c.k.r2dy;
    c.cls.r2dz = (float)c.k.r2dz;
    c.cls.DD = (float)c.k.DD;
    return FSL_OK;
}

// errors of one judgement from the per-row sums (a = MLP, b = dynamic)
void judge_errors(const std::vector<double> &rows, int H, double *perr, double *cerr)
{
    double num = 0, den = 0, d2 = 0, b2 = 0;
    for (int j = 0; j < H; j++) {
        const double a = rows[4 * j], b = rows[4 * j + 1];
        num += (a - b) * (a - b);
        den += b * b;
        d2 += rows[4 * j + 2];
        b2 += rows[4 * j + 3];
    }
    *perr = den > 0 ? std::sqrt(num / den) : (num > 0 ? INFINITY : 0.0);
    *cerr = b2 > 0 ? std::sqrt(d2 / b2) : (d2 > 0 ? INFINITY : 0.0);
}

int check_tc_error(Ctx &c)
{
    int herr = 0;
    if (cudaMemcpyAsync(&herr, c.cl_err, sizeof(int), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    if (herr) {
        c.err = "tensor-core closure kernel: bounded wait gave up";
        return FSL_ERR_TIMEOUT;
    }
    return FSL_OK;
}

// One judgement on U^n (ghost layer filled): the dynamic procedure into c.mu
// and c.cd32, the MLP into the alternate viscosity buffer and c.cs2_32, and
// the plane-averaged comparisons.  Sets c.last_perr / last_cerr (Cs^2) and
// c.last_merr (SGS viscosity profile) and c.last_verr (SGS viscosity profile
// against the effective viscosity mu_L + <mu_dyn>).
int judge_now(Ctx &c)
{
    const bool fp32 = c.p.precision == FSL_PREC_FP32;
    const int H = c.g.H;
    // the dynamic procedure in the path's own precision: mu into c.mu / c.mu32
    if (fp32) launch_dynsmag32(c, c.U, c.cd32);
    else launch_dynsmag(c, c.U, c.cd32);
    if (launch_closure_infer(c, c.U, fp32 ? nullptr : c.mu_alt, fp32 ? c.mu32_alt : nullptr, c.cs2_32, c.cl_params,
                             c.cl_err))
        return FSL_ERR_CUDA;
    launch_judge_rows(c, c.cs2_32, c.cd32, c.judge_rows);
    if (fp32) launch_judge_rows(c, c.mu32_alt, c.mu32, c.judge_rows + 4 * H);
    else launch_judge_rows(c, c.mu_alt, c.mu, c.judge_rows + 4 * H);
    std::vector<double> rows(8 * (size_t)H);
    if (cudaMemcpyAsync(rows.data(), c.judge_rows, rows.size() * sizeof(double), cudaMemcpyDeviceToHost,
                        c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    int rc = check_tc_error(c);
    if (rc) return rc;
    judge_errors(rows, H, &c.last_perr, &c.last_cerr);
    std::vector<double> mrows(rows.begin() + 4 * H, rows.end());
    double mcell;
    judge_errors(mrows, H, &c.last_merr, &mcell);
    // rows j in [3, H-2] hold sums over the (L-4)(D-4) band cells of the plane
    const double nb = (double)(c.g.L - 4) * (c.g.D - 4);
    double num = 0, den = 0, anum = 0, aden = 0, ratio = 0;
    int active = 0;
    for (int j = 2; j <= H - 3; j++) {
        const double a = mrows[4 * j] / nb, b = mrows[4 * j + 1] / nb;
        num += (a - b) * (a - b);
        den += (c.p.mu_L + b) * (c.p.mu_L + b);
        ratio = std::max(ratio, b / c.p.mu_L);
        if (b >= c.judge_floor * c.p.mu_L) { // the SGS model acts on this row
            anum += (a - b) * (a - b);
            aden += b * b;
            active++;
        }
    }
    c.last_verr = den > 0 ? std::sqrt(num / den) : (num > 0 ? INFINITY : 0.0);
    c.last_aerr = active ? std::sqrt(anum / aden) : 0.0;
    c.last_dyn_ratio = ratio;
    c.last_active_rows = active;
    return FSL_OK;
}

// Both criteria of a judgement: the effective viscosity over all rows, and
// the SGS viscosity itself over the rows where the dynamic model acts.  NaN
// errors fail.
bool judge_passes(const Ctx &c)
{
    if (!(c.last_verr <= c.judge_thr)) return false;
    if (c.last_active_rows > 0 && !(c.last_aerr <= c.judge_thr_active)) return false;
    return true;
}

} // namespace

namespace fsl {

// SGS viscosity of one step under FSL_SGS_LEARNED (called after the ghost fill
// of U^n).  Writes c.mu (FP64 path) or c.mu32 (FP32 path).
int closure_step_sgs(Ctx &c)
{
    if (!c.cl_alloc || !c.cl_weights) {
        c.err = "learned closure selected but no weights set (fsl_closure_set_weights)";
        return FSL_ERR_ARG;
    }
    const bool fp32 = c.p.precision == FSL_PREC_FP32;
    const bool judge = c.judge_every > 0 && ((c.step - 1) % (unsigned)c.judge_every == 0);
    if (judge) {
        int rc = judge_now(c);
        if (rc) return rc;
        c.judgements++;
        c.last_judge_step = c.step;
        const bool fail_ = !judge_passes(c);
        if (fail_ && !c.using_dynamic) c.fallbacks++;
        c.using_dynamic = fail_;
        if (fail_) c.dynamic_steps++; // judge_now left the dynamic viscosity in place
        const size_t fs = (size_t)c.g.fstride;
        if (!c.using_dynamic) {
            if (fp32) cudaMemcpyAsync(c.mu32, c.mu32_alt, fs * sizeof(float), cudaMemcpyDeviceToDevice, c.stream);
            else cudaMemcpyAsync(c.mu, c.mu_alt, fs * sizeof(double), cudaMemcpyDeviceToDevice, c.stream);
        }
        return FSL_OK;
    }
    if (c.using_dynamic) {
        if (fp32) launch_dynsmag32(c, c.U);
        else launch_dynsmag(c, c.U);
        c.dynamic_steps++;
        return FSL_OK;
    }
    if (launch_closure_infer(c, c.U, fp32 ? nullptr : c.mu, fp32 ? c.mu32 : nullptr, nullptr, c.cl_params,
                             c.cl_err))
        return FSL_ERR_CUDA;
    return FSL_OK;
}

int closure_ensure(Ctx &c) { return ensure_closure(c); }

void closure_free(Ctx &c)
{
    if (!c.cl_alloc) return;
    cudaFree(c.cl_params); cudaFree(c.cd32); cudaFree(c.cs2_32); cudaFree(c.cl_err); cudaFree(c.cl_vel); cudaFree(c.judge_rows);
    cudaFree(c.mu_alt); cudaFree(c.mu32_alt);
    c.cl_alloc = false;
}

} // namespace fsl

extern "C" {

int fsl_closure_set_scales(fsl_ctx *h, double t_ref, double len_ref)
{
    if (!h) return FSL_ERR_ARG;
    return set_scales(h->c, t_ref, len_ref);
}

int fsl_closure_set_weights(fsl_ctx *h, const float *params)
{
    if (!h || !params) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_closure(c);
    if (rc) return rc;
    if (c.cls.DD == 0.f) set_scales(c, 1.0, 1.0);
    if (cudaMemcpyAsync(c.cl_params, params, kNParams * sizeof(float), cudaMemcpyHostToDevice, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    c.cl_weights = true;
    return FSL_OK;
}

int fsl_closure_get_weights(fsl_ctx *h, float *params)
{
    if (!h || !params || !h->c.cl_weights) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (cudaMemcpyAsync(params, c.cl_params, kNParams * sizeof(float), cudaMemcpyDeviceToHost, c.stream) !=
            cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    return FSL_OK;
}

int fsl_closure_judge(fsl_ctx *h, int every, double threshold)
{
    if (!h || every < 0 || !(threshold >= 0)) return FSL_ERR_ARG;
    h->c.judge_every = every;
    h->c.judge_thr = threshold;
    return FSL_OK;
}

int fsl_closure_judge_active(fsl_ctx *h, double floor, double threshold)
{
    if (!h || !(floor > 0) || !(threshold >= 0)) return FSL_ERR_ARG;
    h->c.judge_floor = floor;
    h->c.judge_thr_active = threshold;
    return FSL_OK;
}

int fsl_closure_get_stats(fsl_ctx *h, fsl_closure_stats *s)
{
    if (!h || !s) return FSL_ERR_ARG;
    const Ctx &c = h->c;
    memset(s, 0, sizeof *s);
    s->mu_active_err = c.last_aerr;
    s->dyn_ratio = c.last_dyn_ratio;
    s->active_rows = c.last_active_rows;
    s->dynamic_steps = c.dynamic_steps;
    s->profile_err = c.last_perr;
    s->mu_profile_err = c.last_merr;
    s->cell_err = c.last_cerr;
    s->visc_err = c.last_verr;
    s->judgements = c.judgements;
    s->fallbacks = c.fallbacks;
    s->using_dynamic = c.using_dynamic ? 1 : 0;
    s->last_step = c.last_judge_step;
    return FSL_OK;
}

int fsl_closure_compare(fsl_ctx *h, float *cs2_mlp, float *cs2_dyn, fsl_closure_stats *errs)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (!c.cl_alloc || !c.cl_weights) return FSL_ERR_ARG;
    int rc = 0;
    launch_ghost(c, c.U);
    if ((rc = ensure_dyn_scratch(c))) return rc;
    if ((rc = judge_now(c))) return rc;
    if (errs) fsl_closure_get_stats(h, errs);
    const Grid &g = c.g;
    for (int which = 0; which < 2; which++) {
        float *dst = which ? cs2_dyn : cs2_mlp;
        const float *src = which ? c.cd32 : c.cs2_32;
        if (!dst) continue;
        if (cudaMemcpy2DAsync(dst, (g.D + 2) * sizeof(float), src + g.off, g.pk * sizeof(float),
                              (g.D + 2) * sizeof(float), (size_t)(g.L + 2) * (g.H + 2), cudaMemcpyDeviceToHost,
                              c.stream) != cudaSuccess)
            return FSL_ERR_CUDA;
    }
    return cudaStreamSynchronize(c.stream) == cudaSuccess ? FSL_OK : FSL_ERR_CUDA;
}

// ---- trainer -------------------------------------------------------------------

int fsl_trainer_create(long long capacity, unsigned long long seed, fsl_trainer **out)
{
    if (!out || capacity < 128) return FSL_ERR_ARG;
    *out = nullptr;
    fsl_trainer *t = new (std::nothrow) fsl_trainer();
    if (!t) return FSL_ERR_NOMEM;
    t->cap = capacity;
    t->seed = seed;
    bool ok = cudaStreamCreateWithFlags(&t->st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->X, (size_t)capacity * 8 * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->Y, (size_t)capacity * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->P, kNParams * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->M, kNParams * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->V, kNParams * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->Gpart, (size_t)t->maxblk * kNParams * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->Gout, kNParams * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->lossp, t->maxblk * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc((void **)&t->err, sizeof(int)) == cudaSuccess;
    if (!ok) {
        fsl_trainer_destroy(t);
        return FSL_ERR_NOMEM;
    }
    std::vector<float> p;
    init_params(p, seed);
    cudaMemcpy(t->P, p.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemset(t->M, 0, kNParams * sizeof(float));
    cudaMemset(t->V, 0, kNParams * sizeof(float));
    cudaMemset(t->err, 0, sizeof(int));
    *out = t;
    return FSL_OK;
}

int fsl_trainer_destroy(fsl_trainer *t)
{
    if (!t) return FSL_ERR_ARG;
    if (t->st) cudaStreamSynchronize(t->st);
    cudaFree(t->X); cudaFree(t->Y); cudaFree(t->P); cudaFree(t->M); cudaFree(t->V);
    cudaFree(t->Gpart); cudaFree(t->Gout); cudaFree(t->lossp); cudaFree(t->err);
    if (t->st) cudaStreamDestroy(t->st);
    delete t;
    return FSL_OK;
}

int fsl_trainer_harvest(fsl_trainer *t, fsl_ctx *h, int stride)
{
    if (!t || !h || stride < 1) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc = ensure_closure(c);
    if (rc) return rc;
    if (c.cls.DD == 0.f) return FSL_ERR_ARG; // fsl_closure_set_scales first
    if ((rc = ensure_dyn_scratch(c))) return rc;
    launch_ghost(c, c.U);
    launch_dynsmag(c, c.U, c.cd32);
    if (c.g.L < 5 || c.g.H < 5 || c.g.D < 5) return FSL_ERR_ARG;
    const long long ncell = (long long)(c.g.L - 4) * (c.g.H - 4) * (c.g.D - 4);
    const long long offset = ((long long)c.step * 7919LL) % stride;
    const long long nsamp = (ncell - offset + stride - 1) / stride;
    launch_harvest(c, c.cd32, stride, offset, t->X, t->Y, t->cap, t->n);
    if (cudaStreamSynchronize(c.stream) != cudaSuccess) return FSL_ERR_CUDA;
    t->n = std::min(t->cap, t->n + nsamp);
    t->shuffled = false;
    t->inv_wmean = 0.f;
    return FSL_OK;
}

long long fsl_trainer_size(fsl_trainer *t) { return t ? t->n : -1; }

int fsl_trainer_get_samples(fsl_trainer *t, float *X, float *Y, long long n)
{
    if (!t || n < 0 || n > t->n) return FSL_ERR_ARG;
    if (X && cudaMemcpy(X, t->X, (size_t)n * 8 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return FSL_ERR_CUDA;
    if (Y && cudaMemcpy(Y, t->Y, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return FSL_ERR_CUDA;
    return FSL_OK;
}

int fsl_trainer_set_samples(fsl_trainer *t, const float *X, const float *Y, long long n)
{
    if (!t || !X || !Y || n < 0 || n > t->cap) return FSL_ERR_ARG;
    if (cudaMemcpy(t->X, X, (size_t)n * 8 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(t->Y, Y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return FSL_ERR_CUDA;
    t->n = n;
    t->shuffled = false;
    t->inv_wmean = 0.f;
    return FSL_OK;
}

int fsl_trainer_set_loss(fsl_trainer *t, int mode)
{
    if (!t || mode < 0 || mode > 1) return FSL_ERR_ARG;
    t->loss_mode = mode;
    return FSL_OK;
}

int fsl_trainer_get_weights(fsl_trainer *t, float *params)
{
    if (!t || !params) return FSL_ERR_ARG;
    return cudaMemcpy(params, t->P, kNParams * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess ? FSL_OK
                                                                                                    : FSL_ERR_CUDA;
}

int fsl_trainer_set_weights(fsl_trainer *t, const float *params)
{
    if (!t || !params) return FSL_ERR_ARG;
    if (cudaMemcpy(t->P, params, kNParams * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return FSL_ERR_CUDA;
    cudaMemset(t->M, 0, kNParams * sizeof(float));
    cudaMemset(t->V, 0, kNParams * sizeof(float));
    t->adam_t = 0;
    return FSL_OK;
}

// 1 / mean of the sample weights (rho |S| t_ref)^2 over the current samples
static int trainer_weights(fsl_trainer *t)
{
    if (t->loss_mode == 0 || t->inv_wmean > 0.f) return FSL_OK;
    std::vector<float> X((size_t)t->n * 8);
    if (cudaMemcpy(X.data(), t->X, X.size() * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return FSL_ERR_CUDA;
    double s = 0;
    for (long long m = 0; m < t->n; m++) {
        const double st = std::expm1((double)X[m * 8]) * X[m * 8 + 6];
        s += st * st;
    }
    const double mean = t->n ? s / (double)t->n : 0.0;
    t->inv_wmean = mean > 0 ? (float)(1.0 / mean) : 1.f;
    return FSL_OK;
}

static int trainer_pass(fsl_trainer *t, const float *X, const float *Y, long long n, float lr, double *loss)
{
    if (trainer_weights(t)) return FSL_ERR_CUDA;
    const float iw = t->loss_mode ? t->inv_wmean : 0.f;
    const long long ntile = (n + 127) / 128;
    const int tpb = (int)((ntile + t->maxblk - 1) / t->maxblk);
    int nblk = 0;
    if (launch_train_grad(t->st, X, Y, n, tpb, t->P, t->Gpart, t->lossp, t->err, &nblk, iw)) return FSL_ERR_CUDA;
    float b1t = 1.f, b2t = 1.f;
    if (lr > 0.f) {
        t->adam_t++;
        b1t = (float)std::pow(0.9, (double)t->adam_t);
        b2t = (float)std::pow(0.999, (double)t->adam_t);
    }
    launch_reduce_adam(t->st, t->Gpart, nblk, t->P, t->M, t->V, t->Gout, lr, b1t, b2t);
    if (loss) {
        std::vector<float> lp(nblk);
        if (cudaMemcpyAsync(lp.data(), t->lossp, nblk * sizeof(float), cudaMemcpyDeviceToHost, t->st) !=
                cudaSuccess ||
            cudaStreamSynchronize(t->st) != cudaSuccess)
            return FSL_ERR_CUDA;
        double s = 0;
        for (float v : lp) s += v;
        *loss = s / (double)n;
    }
    int herr = 0;
    cudaMemcpyAsync(&herr, t->err, sizeof(int), cudaMemcpyDeviceToHost, t->st);
    if (cudaStreamSynchronize(t->st) != cudaSuccess) return FSL_ERR_CUDA;
    return herr ? FSL_ERR_TIMEOUT : FSL_OK;
}

int fsl_trainer_gradient(fsl_trainer *t, long long n, float *grad, double *loss)
{
    if (!t || n < 1 || n > t->n) return FSL_ERR_ARG;
    int rc = trainer_pass(t, t->X, t->Y, n, 0.f, loss);
    if (rc) return rc;
    if (grad && cudaMemcpy(grad, t->Gout, kNParams * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return FSL_ERR_CUDA;
    return FSL_OK;
}

int fsl_trainer_train(fsl_trainer *t, int epochs, long long batch, double lr, double *loss)
{
    if (!t || epochs < 0 || batch < 128 || !(lr > 0) || t->n < batch) return FSL_ERR_ARG;
    batch = (batch / 128) * 128;
    if (!t->shuffled) { // one seeded Fisher-Yates shuffle of the harvested samples
        std::vector<float> X((size_t)t->n * 8), Y((size_t)t->n);
        if (fsl_trainer_get_samples(t, X.data(), Y.data(), t->n)) return FSL_ERR_CUDA;
        uint64_t s = t->seed ^ 0x5DEECE66DULL;
        for (long long i = t->n - 1; i > 0; i--) {
            const long long j = (long long)(splitmix(s) % (uint64_t)(i + 1));
            std::swap(Y[i], Y[j]);
            for (int q = 0; q < 8; q++) std::swap(X[i * 8 + q], X[j * 8 + q]);
        }
        if (fsl_trainer_set_samples(t, X.data(), Y.data(), t->n)) return FSL_ERR_CUDA;
        t->shuffled = true;
    }
    const long long nb = t->n / batch;
    for (int e = 0; e < epochs; e++)
        for (long long b = 0; b < nb; b++) {
            int rc = trainer_pass(t, t->X + b * batch * 8, t->Y + b * batch, batch, (float)lr, nullptr);
            if (rc) return rc;
        }
    return fsl_trainer_gradient(t, t->n, nullptr, loss);
}

} // extern "C"
