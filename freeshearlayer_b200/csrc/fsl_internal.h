// fsl_internal.h -- device layout, context and launcher declarations shared
// by the translation units of libfsl_gpu.so.  Not part of the C ABI.
#pragma once

#include <atomic>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <string>
#include <vector>

#include "../../include/fsl_gpu.h"
#include "fsl_mlp.h"

namespace fsl {

// Padded cell field layout in HBM: (LEN+2)(HIG+2) rows of pk elements, k
// fastest, element (0,0,0) at `off`.  pk is a multiple of 32 bytes' worth of
// elements and off = that multiple - 1, so interior rows (k = 1..DEP) start on
// a 32-byte sector boundary and full rows are read with aligned, coalesced
// sectors.  Fields of one kind sit `fstride` elements apart in one allocation.
struct Grid {
    int L, H, D;
    int pk;
    long long pi;      // elements between i planes = pk * (H+2)
    long long off;     // offset of (0,0,0)
    long long fstride; // elements between fields (multiple of 64)
    __host__ __device__ __forceinline__ long long idx(int i, int j, int k) const
    {
        return off + (long long)i * pi + (long long)j * pk + k;
    }
};

Grid make_grid(int L, int H, int D, int elem_bytes);

// Physical and derived constants of one domain (src/initialize.c:67-94).
struct Consts {
    double rdx, rdy, rdz, r2dx, r2dy, r2dz, r4dx, r4dy, r4dz;
    double mu_L, lambda_L, cp_Pr_T, DD, maxCoNum;
    double CsDD; // Cs DD, the static Smagorinsky factor (src/initialize.c:94)
    double deltaX, deltaY, deltaZ;
    int setup, BL_HIG, cfl_mode, nStages;
};

// Device-resident scalars updated by the time-step reduction.
struct DevScalars {
    double dt, dtx, dty, dtz;
    double maxCo;
    unsigned int status; // bit 0: non-finite or non-positive Courant max; bit 1: non-positive density
    unsigned int pad;
    // Courant maximum of the state written by the last fused stage 3 (bit
    // pattern of a non-negative double, accumulated with atomicMax)
    unsigned long long co_bits;
};

// Disturbance block of one step (host RNG state, src/layer2.c:152-162).
struct Disturb {
    unsigned k_min, k_max;
    double Ud, Vd, Wd;
};

// Dense face arrays (reference face index ranges).
struct Faces {
    double *x[2][5], *y[2][5], *z[2][5];
};

// Outer states of the domain-boundary faces for the fused stage kernel (the
// reference's BounCondOnInterfaces values): x0/xL [5][HIG][DEP] (minus side of
// x face 0, plus side of x face LEN), y0/yH [5][LEN][DEP], z0/zD [5][LEN][HIG].
struct BFaces {
    double *x0, *xL, *y0, *yH, *z0, *zD;
};
struct BFaces32 {
    float *x0, *xL, *y0, *yH, *z0, *zD;
};

// Scratch of the dynamic Smagorinsky procedure (padded layout, FP64).
// Scratch of the fused dynamic procedure (fsl_dyn.cuh, sequence_fused)
template <typename T> struct DynFields {
    T *vel; // 3 fields u, v, w
    T *F;   // 9 fields: the filtered velocities and products; zero where no pass writes
    T *A;   // 6 fields |S| S_ij, ghost layer kept zero
    T *S;   // 1 field |S|
};
typedef DynFields<double> DynScratch;
typedef DynFields<float> DynScratch32;

struct Ctx {
    fsl_params p;
    Consts k;
    Grid g;
    cudaStream_t stream = nullptr;
    int device = 0;
    int sms = 148; // streaming multiprocessors of the device
    // cell fields (FP64): U^n, stage buffer, second stage buffer, mu_SGS
    double *U = nullptr, *Up = nullptr, *Uq = nullptr, *mu = nullptr;
    int cur = 0; // 0: U*_ = U, 1: U*_ = Up
    Faces f{};
    bool faces_alloc = false;
    DynScratch dyn{};
    DynScratch32 dyn32{}; // the FP32 path's own (a shared buffer would mix the two views' zero bands)
    bool dyn_alloc = false;
    BFaces bf{};
    bool bf_alloc = false;
    // FP32-bulk path
    BFaces32 bf32{};
    float *mu32 = nullptr;
    bool fp32_alloc = false;
    int stage_tje = 16; // rows per fused-stage ring tile (incl. the two halo rows); 0: full-lane tile (FP32)
    int stage_seg = 32; // x planes per fused-stage block (fsl_init: 48 for FP32 bulk)
    // learned closure
    ClosureScales cls{};
    float *cl_params = nullptr; // FP32 parameter vector (kNParams)
    float *cd32 = nullptr;      // dynamic-procedure Cs^2, padded FP32
    float *cs2_32 = nullptr;    // closure Cs^2, padded FP32
    double *mu_alt = nullptr;   // closure mu on judgement steps (FP64 path)
    float *mu32_alt = nullptr;  // closure mu on judgement steps (FP32 path)
    int *cl_err = nullptr;      // device error flag of the tensor-core kernels
    float *cl_vel = nullptr;    // FP32 velocities of the padded cells (closure features), 3 fields
    bool vel_fresh = false;     // cl_vel holds U's velocities (the last stage wrote them): no velocity pass
    double *judge_rows = nullptr; // [2][HIG][4] plane sums of the judgement (Cs^2, mu_SGS)
    bool cl_alloc = false, cl_weights = false;
    int infer_poly = 2;         // closure inference: SiLU pairs of 8 on the FMA-pipe tanh (0, 2, 3, 4)
    int judge_every = 100;
    double judge_thr = 0.05;
    bool using_dynamic = false;
    int judgements = 0, fallbacks = 0, dynamic_steps = 0;
    double judge_floor = 0.1, judge_thr_active = 0.4; // SGS-active rows: <mu_dyn> >= floor mu_L
    double last_perr = -1, last_cerr = -1, last_merr = -1, last_verr = -1;
    double last_aerr = -1, last_dyn_ratio = -1;
    int last_active_rows = 0;
    unsigned last_judge_step = 0;
    DevScalars *ds = nullptr; // device scalars
    DevScalars *hs = nullptr; // pinned host mirror
    double *partials = nullptr;
    int npartials = 0;
    double *stage_host = nullptr; // pinned staging for state transfer
    double *stage_dev = nullptr;
    // asynchronous state transfer (fsl_*_state_async): own staging buffers,
    // copy streams (one per direction) and the events that order them
    // against the context's stream
    bool xfer_alloc = false;
    double *xin = nullptr, *xout = nullptr;
    cudaStream_t up = nullptr, down = nullptr;
    cudaEvent_t ev_in_ready = nullptr, ev_in_free = nullptr, ev_out_ready = nullptr, ev_out_free = nullptr;
    // host driver state
    double X = 0;
    int counter = 0;
    unsigned step = 0;
    Disturb dist{};
    // device sums of the probe columns (fsl_favre_*): [station][rho, rho u][HIG]
    double *favre = nullptr;
    int favre_count = 0;
    // the device Courant maximum (DevScalars::co_bits) belongs to the current U^n
    bool co_valid = false;
    // planes (1-based) whose cells enter the Courant maximum; 1..L unless an
    // x-slab of a decomposed domain restricts it to the planes it owns
    int co_i0 = 1, co_i1 = 0;
    // fsl_step_stage: the stage the step in progress runs next (2 or 3), or 0
    // between steps; the current stage state is then in Up (2) or Uq (3)
    int stage_next = 0;
    double dt_host = 0; // host copy of dt, valid after sync
    double maxco_host = 0;
    unsigned long long bytes = 0;
    std::string err;
    // profiler: event pairs per kernel class, launch counters
    bool prof = false;
    struct Rec {
        int cls;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> evpool;
    double kms[FSL_K_COUNT] = {0};
    unsigned long long klaunch[FSL_K_COUNT] = {0};
    int open_cls = -1;
    cudaEvent_t open_ev = nullptr;
};

// Bracket a group of launches of one kernel class (no-ops unless profiling).
void prof_begin(Ctx &c, int cls);
void prof_end(Ctx &c, int cls, int nkernels);

int ensure_dyn_scratch(Ctx &c);  // SGS scratch of the dynamic procedure + the FP32 SGS field (fsl_api.cu)
int step_prelude32(Ctx &c);      // an FP32-bulk step up to its first stage (fsl_api.cu)
int closure_step_sgs(Ctx &c);    // SGS of one step under FSL_SGS_LEARNED (fsl_closure.cu)
int closure_ensure(Ctx &c);
void closure_free(Ctx &c);

// An NVTX range named for a C-ABI entry point, open for the call (host side:
// profilers attribute the call's launches to it; without a profiler attached
// a push/pop is a check of a null hook).
struct ApiRange {
    explicit ApiRange(const char *name) { nvtxRangePushA(name); }
    ~ApiRange() { nvtxRangePop(); }
    ApiRange(const ApiRange &) = delete;
    ApiRange &operator=(const ApiRange &) = delete;
};

// A kernel's dynamic shared-memory limit, raised once per device (the
// attribute holds for the device that is current when it is set, and one
// process may drive several devices).  false if the runtime refuses it.
inline bool smem_limit_once(const void *kernel, size_t smem, std::atomic<uint64_t> &done)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    const uint64_t bit = 1ull << dev;
    if (done.load() & bit) return true;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return false;
    done.fetch_or(bit);
    return true;
}

// ---- launchers (fsl_phase.cu) ------------------------------------------------
void launch_ghost(Ctx &c, double *cur);
void launch_recon(Ctx &c, const double *cur);
void launch_ifbc(Ctx &c, const Disturb &d);
void launch_fluxes(Ctx &c, const double *cur);
void launch_evolution(Ctx &c, int nstages, int stage);
void launch_dynsmag(Ctx &c, const double *U, float *cd = nullptr); // cd: optional Cs^2 output
// the same procedure in FP32 (the FP32-bulk path): mu_SGS into c.mu32
void launch_dynsmag32(Ctx &c, const double *U, float *cd = nullptr);
void launch_judge_rows(Ctx &c, const float *a, const float *b, double *rows);
void launch_judge_rows(Ctx &c, const float *a, const double *b, double *rows);
void launch_judge_rows(Ctx &c, const double *a, const double *b, double *rows);
void launch_courant(Ctx &c);
// dt update from the Courant maximum the fused stage 3 accumulated
void launch_courant_apply(Ctx &c);
void launch_state_scatter(Ctx &c, double *dst, const double *packed, int i0, int ni);
void launch_state_gather(Ctx &c, const double *src, double *packed, int i0, int ni);
void launch_courant_to_bits(Ctx &c);
void launch_sums(Ctx &c, const double *U, int i0, int ni, double *out5);
void launch_plane_sums(Ctx &c, const double *U, int i0, int ni, double *rows);

// ---- fused path (fsl_fused.cu) ----------------------------------------------
void launch_bface(Ctx &c, const double *cur, const Disturb &d);
// One RK3 stage: cur (ghosts filled) -> out; un = U^n.
int launch_stage(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant = false);
// FP32-bulk variants (fsl_fused32.cu): boundary states in bf32, SGS viscosity in mu32.
void launch_bface32(Ctx &c, const double *cur, const Disturb &d);
// vel (full-lane tile, temporal setup, stage 3 only): also write the FP32
// velocities of `out` into that field (the closure's feature velocities)
int launch_stage32(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant = false,
                   float *vel = nullptr);
// The three stages of an FP32-bulk step of several domains in one persistent
// cooperative launch (fsl_fused32.cu); opaque plan built per member set.
struct WidePlan;
int wide_plan_build(const std::vector<Ctx *> &members, WidePlan **plan, std::string &why);
void wide_plan_free(WidePlan *plan);
int wide_plan_launch(WidePlan *plan, cudaStream_t st);
int wide_plan_set_limit(WidePlan *plan, unsigned polls);
int wide_plan_check(WidePlan *plan, cudaStream_t st); // FSL_ERR_TIMEOUT (and reset) after a barrier gave up

// ---- learned closure (fsl_mlp.cu) ---------------------------------------------
int launch_closure_infer(Ctx &c, const double *U, double *mu64, float *mu32, float *cs2_out, const float *P,
                         int *err);
void launch_harvest(Ctx &c, const float *cd, long long stride, long long offset, float *X, float *Y, long long cap,
                    long long base);
int launch_train_grad(cudaStream_t st, const float *X, const float *Y, long long n, int tpb, const float *P,
                      float *Gpart, float *loss_part, int *err, int *nblk_out, float inv_wmean);
void launch_reduce_adam(cudaStream_t st, const float *Gpart, int nblk, float *P, float *M, float *V, float *Gout,
                        float lr, float b1t, float b2t);

} // namespace fsl

// The opaque handle of the C ABI.
struct fsl_ctx {
    fsl::Ctx c;
};
