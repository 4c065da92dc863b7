// fsl_ensemble.cu -- ensembles of independent shear layers advanced together.
//
// Each member is an ordinary context (its own grid, Mach and Reynolds number,
// seed, stream and buffers).  A step of the ensemble is the members' fused
// steps issued on their own streams, forked from and joined to the
// ensemble's stream; `chunk` such steps are captured once into a CUDA graph
// and the graph is replayed, so a whole chunk of the ensemble is one launch
// and the members' kernels run side by side on the SMs.  Graph replay
// launches exactly the kernels a plain fsl_step would, with the same
// arguments, so every member's result is bit-identical to stepping it alone.
//
// What a graph may not hold decides what members may be: temporal setup
// (the spatial inflow disturbance is redrawn on the host every step),
// closure judgements off (a judgement reads its errors back to the host),
// profiling off.  The Courant maximum of each member's last stage feeds the
// next step on the device (DevScalars::co_bits), so no step needs the host.
#include <algorithm>
#include <vector>

#include "fsl_internal.h"

using namespace fsl;

struct fsl_ensemble {
    std::vector<fsl_ctx *> m;
    cudaStream_t stream = nullptr;
    std::vector<cudaEvent_t> fork, join;         // ordering outside graphs
    std::vector<cudaEvent_t> cap_fork, cap_join; // fork/join inside a capture
    cudaGraphExec_t exec = nullptr;
    int exec_steps = 0;      // steps captured in exec (0: none)
    unsigned long long gen = 0, exec_gen = ~0ull; // member configuration generation
    int chunk = 10;
    std::string err;
    // the persistent path: the members' three stages of a step in one
    // cooperative launch (all members FP32 bulk, reference reconstruction,
    // full-lane tiles); otherwise each member's fused steps
    WidePlan *plan = nullptr;
    unsigned long long plan_gen = ~0ull;
    bool persistent_off = false; // the persistent path could not be captured here
    unsigned barrier_limit = 1u << 24;
    std::string why_not;
    std::vector<int> sig; // the members' launch shapes the captured work was built for
};

namespace {

int ens_fail(fsl_ensemble *e, int code, const char *what)
{
    e->err = what;
    return code;
}

void drop_graph(fsl_ensemble *e)
{
    if (e->exec) cudaGraphExecDestroy(e->exec);
    e->exec = nullptr;
    e->exec_steps = 0;
}

int check_member(fsl_ensemble *e, const Ctx &c)
{
    if (c.p.setup != FSL_SETUP_TEMPORAL)
        return ens_fail(e, FSL_ERR_UNSUPPORTED, "ensemble members need the temporal setup");
    if (c.p.nStages != 3) return ens_fail(e, FSL_ERR_UNSUPPORTED, "ensemble members need nStages = 3");
    if (c.p.sgs == FSL_SGS_LEARNED && c.judge_every > 0)
        return ens_fail(e, FSL_ERR_UNSUPPORTED, "ensemble members with the learned closure need judgements off");
    if (c.prof) return ens_fail(e, FSL_ERR_UNSUPPORTED, "ensemble members must not be profiling");
    if (c.co_i0 != 1 || c.co_i1 != c.p.LEN)
        return ens_fail(e, FSL_ERR_UNSUPPORTED, "ensemble members must be whole domains, not x-slabs");
    if (c.stage_next != 0) return ens_fail(e, FSL_ERR_ARG, "an ensemble member is in the middle of a step");
    return FSL_OK;
}

// The persistent plan for the current members, when they all qualify.
void refresh_plan(fsl_ensemble *e)
{
    if (e->plan && e->plan_gen == e->gen) return;
    wide_plan_free(e->plan);
    e->plan = nullptr;
    if (e->persistent_off) return;
    std::vector<Ctx *> ms;
    for (fsl_ctx *h : e->m) ms.push_back(&h->c);
    WidePlan *p = nullptr;
    if (wide_plan_build(ms, &p, e->why_not) == FSL_OK) {
        wide_plan_set_limit(p, e->barrier_limit);
        e->plan = p;
        e->why_not.clear();
    }
    e->plan_gen = e->gen;
}

// Capture `steps` persistent-path steps: per step the members' work before
// their first stage (each on its own stream), then one cooperative launch
// of all members' three stages.
int capture_persistent(fsl_ensemble *e, int steps)
{
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return ens_fail(e, FSL_ERR_CUDA, "cudaStreamBeginCapture");
    int rc = FSL_OK;
    for (int t = 0; t < steps && !rc; t++) {
        cudaEventRecord(e->cap_fork[0], e->stream);
        for (size_t q = 0; q < e->m.size(); q++) {
            Ctx &c = e->m[q]->c;
            cudaStreamWaitEvent(c.stream, e->cap_fork[0], 0);
            if (!rc) rc = step_prelude32(c);
            cudaEventRecord(e->cap_join[q], c.stream);
            cudaStreamWaitEvent(e->stream, e->cap_join[q], 0);
        }
        if (!rc) rc = wide_plan_launch(e->plan, e->stream);
        for (fsl_ctx *h : e->m) h->c.co_valid = true;
    }
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
    for (fsl_ctx *h : e->m) h->c.step -= (unsigned)steps;
    if (rc || ce != cudaSuccess || !graph) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError(); // a refused capture leaves no sticky state
        return rc ? rc : FSL_ERR_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        e->exec = nullptr;
        cudaGetLastError();
        return FSL_ERR_CUDA;
    }
    e->exec_steps = steps;
    e->exec_gen = e->gen;
    return FSL_OK;
}

// Capture `steps` fused steps of every member into one graph.
int capture(fsl_ensemble *e, int steps)
{
    drop_graph(e);
    refresh_plan(e);
    if (e->plan) {
        const int rc = capture_persistent(e, steps);
        if (rc == FSL_OK) return FSL_OK;
        // the cooperative launch could not be captured: the members' fused
        // steps instead, from now on
        drop_graph(e);
        e->persistent_off = true;
        wide_plan_free(e->plan);
        e->plan = nullptr;
        e->why_not = "the cooperative stage launch could not be captured in a graph";
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return ens_fail(e, FSL_ERR_CUDA, "cudaStreamBeginCapture");
    int rc = FSL_OK;
    // one fork, each member's `steps` steps in order on its own stream, one
    // join: members never wait for one another inside the graph
    cudaEventRecord(e->cap_fork[0], e->stream);
    for (size_t q = 0; q < e->m.size(); q++) {
        Ctx &c = e->m[q]->c;
        cudaStreamWaitEvent(c.stream, e->cap_fork[0], 0);
        if (!rc) rc = fsl_step(e->m[q], steps);
        cudaEventRecord(e->cap_join[q], c.stream);
        cudaStreamWaitEvent(e->stream, e->cap_join[q], 0);
    }
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &graph);
    // the host-side step counters advanced during capture; replays advance them
    for (fsl_ctx *h : e->m) h->c.step -= (unsigned)steps;
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return ens_fail(e, rc, "a member step failed during capture");
    }
    if (ce != cudaSuccess || !graph) return ens_fail(e, FSL_ERR_CUDA, "cudaStreamEndCapture");
    const cudaError_t ie = cudaGraphInstantiate(&e->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
        e->exec = nullptr;
        return ens_fail(e, FSL_ERR_CUDA, "cudaGraphInstantiate");
    }
    e->exec_steps = steps;
    e->exec_gen = e->gen;
    return FSL_OK;
}

int replay(fsl_ensemble *e)
{
    if (cudaGraphLaunch(e->exec, e->stream) != cudaSuccess) return ens_fail(e, FSL_ERR_CUDA, "cudaGraphLaunch");
    for (fsl_ctx *h : e->m) h->c.step += (unsigned)e->exec_steps;
    return FSL_OK;
}

// Member states, device scalars and host driver state, for the autotuner.
struct Snapshot {
    double *U = nullptr;
    DevScalars ds{};
    unsigned step = 0;
    double X = 0;
    int counter = 0, cur = 0;
    Disturb dist{};
    bool co_valid = false;
};

int take(Ctx &c, Snapshot &s)
{
    const size_t bytes = 5 * (size_t)c.g.fstride * sizeof(double);
    if (cudaMalloc((void **)&s.U, bytes) != cudaSuccess) return FSL_ERR_NOMEM;
    if (cudaMemcpyAsync(s.U, c.U, bytes, cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess ||
        cudaMemcpyAsync(&s.ds, c.ds, sizeof(DevScalars), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    s.step = c.step; s.X = c.X; s.counter = c.counter; s.cur = c.cur; s.dist = c.dist; s.co_valid = c.co_valid;
    return FSL_OK;
}

int restore(Ctx &c, Snapshot &s)
{
    const size_t bytes = 5 * (size_t)c.g.fstride * sizeof(double);
    if (cudaMemcpyAsync(c.U, s.U, bytes, cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess ||
        cudaMemcpyAsync(c.ds, &s.ds, sizeof(DevScalars), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return FSL_ERR_CUDA;
    c.step = s.step; c.X = s.X; c.counter = s.counter; c.cur = s.cur; c.dist = s.dist; c.co_valid = s.co_valid;
    return FSL_OK;
}

} // namespace

extern "C" {

int fsl_ensemble_create(fsl_ctx *const *members, int n, fsl_ensemble **out)
{
    if (!members || n < 1 || !out) return FSL_ERR_ARG;
    *out = nullptr;
    for (int q = 0; q < n; q++) {
        if (!members[q]) return FSL_ERR_ARG;
        for (int r = 0; r < q; r++)
            if (members[r] == members[q]) return FSL_ERR_ARG;
    }
    fsl_ensemble *e = new (std::nothrow) fsl_ensemble();
    if (!e) return FSL_ERR_NOMEM;
    e->m.assign(members, members + n);
    bool ok = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) == cudaSuccess;
    e->fork.resize(1, nullptr);
    e->join.resize(n, nullptr);
    e->cap_fork.resize(1, nullptr);
    e->cap_join.resize(n, nullptr);
    for (auto *v : {&e->fork, &e->join, &e->cap_fork, &e->cap_join})
        for (cudaEvent_t &ev : *v) ok = ok && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        fsl_ensemble_destroy(e);
        return FSL_ERR_CUDA;
    }
    *out = e;
    return FSL_OK;
}

int fsl_ensemble_destroy(fsl_ensemble *e)
{
    if (!e) return FSL_ERR_ARG;
    if (e->stream) cudaStreamSynchronize(e->stream);
    drop_graph(e);
    wide_plan_free(e->plan);
    for (auto *v : {&e->fork, &e->join, &e->cap_fork, &e->cap_join})
        for (cudaEvent_t ev : *v)
            if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return FSL_OK;
}

const char *fsl_ensemble_last_error(const fsl_ensemble *e) { return e ? e->err.c_str() : "no ensemble"; }

void *fsl_ensemble_stream(fsl_ensemble *e) { return e ? (void *)e->stream : nullptr; }

int fsl_ensemble_persistent(fsl_ensemble *e)
{
    if (!e) return FSL_ERR_ARG;
    refresh_plan(e);
    return e->plan ? 1 : 0;
}

int fsl_ensemble_set_barrier_limit(fsl_ensemble *e, unsigned polls)
{
    if (!e) return FSL_ERR_ARG;
    drop_graph(e); // the limit is a launch argument
    e->barrier_limit = polls;
    if (e->plan) wide_plan_set_limit(e->plan, polls);
    return FSL_OK;
}

int fsl_ensemble_set_chunk(fsl_ensemble *e, int steps)
{
    if (!e || steps < 1 || steps > 1000) return FSL_ERR_ARG;
    if (steps != e->chunk) drop_graph(e);
    e->chunk = steps;
    return FSL_OK;
}

// A member retuned after the ensemble captured its work invalidates it.
static void check_shapes(fsl_ensemble *e)
{
    std::vector<int> sig;
    for (fsl_ctx *h : e->m) {
        sig.push_back(h->c.stage_tje);
        sig.push_back(h->c.stage_seg);
    }
    if (sig != e->sig) {
        e->sig = sig;
        e->gen++;
    }
}

int fsl_ensemble_step(fsl_ensemble *e, int nsteps)
{
    ApiRange range_("fsl_ensemble_step");
    if (!e || nsteps < 0) return FSL_ERR_ARG;
    if (nsteps == 0) return FSL_OK;
    int rc;
    for (fsl_ctx *h : e->m)
        if ((rc = check_member(e, h->c))) return rc;
    check_shapes(e);
    // a member whose Courant maximum is not on the device yet (fresh upload,
    // a per-phase call) takes one plain step first: it allocates what the
    // step needs and leaves the graph-ready device state
    bool warm = false;
    for (fsl_ctx *h : e->m) warm = warm || !h->c.co_valid || h->c.cur != 0;
    cudaEventRecord(e->fork[0], e->stream);
    if (warm) {
        for (size_t q = 0; q < e->m.size(); q++) {
            Ctx &c = e->m[q]->c;
            cudaStreamWaitEvent(c.stream, e->fork[0], 0);
            if ((rc = fsl_step(e->m[q], 1))) return ens_fail(e, rc, fsl_last_error(e->m[q]));
            cudaEventRecord(e->join[q], c.stream);
            cudaStreamWaitEvent(e->stream, e->join[q], 0);
        }
        nsteps--;
        drop_graph(e);
    } else {
        // members' own streams must not run ahead of earlier ensemble work
        for (fsl_ctx *h : e->m) cudaStreamWaitEvent(h->c.stream, e->fork[0], 0);
    }
    // previous work on the members' streams precedes the graph
    for (size_t q = 0; q < e->m.size(); q++) {
        cudaEventRecord(e->join[q], e->m[q]->c.stream);
        cudaStreamWaitEvent(e->stream, e->join[q], 0);
    }
    const int full = nsteps / e->chunk, rest = nsteps % e->chunk;
    if (full > 0) {
        if (!e->exec || e->exec_steps != e->chunk || e->exec_gen != e->gen)
            if ((rc = capture(e, e->chunk))) return rc;
        for (int t = 0; t < full; t++)
            if ((rc = replay(e))) return rc;
    }
    if (rest > 0) {
        if ((rc = capture(e, rest))) return rc;
        if ((rc = replay(e))) return rc;
        drop_graph(e); // keep the chunk-sized graph the common case
    }
    // members' streams follow the ensemble's work
    cudaEventRecord(e->fork[0], e->stream);
    for (fsl_ctx *h : e->m) cudaStreamWaitEvent(h->c.stream, e->fork[0], 0);
    return cudaGetLastError() == cudaSuccess ? FSL_OK : ens_fail(e, FSL_ERR_CUDA, "ensemble launch");
}

int fsl_ensemble_sync(fsl_ensemble *e)
{
    if (!e) return FSL_ERR_ARG;
    if (cudaStreamSynchronize(e->stream) != cudaSuccess) return ens_fail(e, FSL_ERR_CUDA, "ensemble stream");
    if (e->plan) {
        const int brc = wide_plan_check(e->plan, e->stream);
        if (brc) return ens_fail(e, brc, "a grid barrier of the persistent stage launch gave up");
    }
    for (fsl_ctx *h : e->m) {
        int rc = fsl_sync(h);
        if (rc) return ens_fail(e, rc, fsl_last_error(h));
    }
    return FSL_OK;
}

// Autotuner of the fused-stage tile shape (rows per tile, x planes per
// block), one shape for all members: each candidate is timed over
// trial_steps graph-replayed ensemble steps after one untimed chunk; member
// states are restored afterwards, so tuning changes no result.
int fsl_ensemble_tune(fsl_ensemble *e, int trial_steps, int *rows_out, int *seg_out, double *best_ms)
{
    if (!e || trial_steps < 1) return FSL_ERR_ARG;
    int rc;
    for (fsl_ctx *h : e->m)
        if ((rc = check_member(e, h->c))) return rc;
    if ((rc = fsl_ensemble_sync(e))) return rc;
    std::vector<Snapshot> snap(e->m.size());
    for (size_t q = 0; q < e->m.size(); q++)
        if ((rc = take(e->m[q]->c, snap[q]))) return ens_fail(e, rc, "tuner snapshot");
    // rows 0: the full-lane persistent tile (FP32 bulk, reference scheme;
    // it balances its own planes, so one planes-per-block value is tried)
    const int rows_c[4] = {0, 8, 12, 16}, seg_c[5] = {8, 16, 32, 48, 64};
    int best_r = e->m[0]->c.stage_tje, best_s = e->m[0]->c.stage_seg;
    double best = 1e300;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    for (int ri = 0; ri < 4 && !rc; ri++)
        for (int si = 0; si < (rows_c[ri] == 0 ? 1 : 5) && !rc; si++) {
            for (fsl_ctx *h : e->m) {
                h->c.stage_tje = rows_c[ri];
                h->c.stage_seg = seg_c[si];
            }
            e->gen++;
            // one plain step per member (sets the kernels' attributes outside
            // any capture), then a captured chunk: one untimed, one timed replay
            if ((rc = fsl_ensemble_sync(e))) break;
            for (fsl_ctx *h : e->m)
                if ((rc = fsl_step(h, 1))) break;
            if (rc || (rc = fsl_ensemble_sync(e))) break;
            if ((rc = capture(e, trial_steps)) || (rc = replay(e))) break;
            cudaEventRecord(a, e->stream);
            if ((rc = replay(e))) break;
            cudaEventRecord(b, e->stream);
            if (cudaEventSynchronize(b) != cudaSuccess) {
                rc = ens_fail(e, FSL_ERR_CUDA, "tuner timing");
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            const double per = ms / trial_steps;
            if (per < best) {
                best = per;
                best_r = rows_c[ri];
                best_s = seg_c[si];
            }
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    drop_graph(e);
    if (!rc) rc = fsl_ensemble_sync(e);
    for (size_t q = 0; q < e->m.size(); q++) {
        Ctx &c = e->m[q]->c;
        c.stage_tje = best_r;
        c.stage_seg = best_s;
        const int r2 = restore(c, snap[q]);
        if (!rc) rc = r2;
        cudaFree(snap[q].U);
    }
    e->gen++;
    if (rc) return rc;
    if (rows_out) *rows_out = best_r;
    if (seg_out) *seg_out = best_s;
    if (best_ms) *best_ms = best;
    return FSL_OK;
}

} // extern "C"
