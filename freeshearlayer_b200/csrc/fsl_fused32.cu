// fsl_fused32.cu -- FP32-bulk instantiation of the fused stage kernel.
//
// Reconstruction, Riemann and viscous fluxes run in FP32 (compiled with
// --use_fast_math: FMA contraction, approximate FP32 division and square
// root); the conserved variables, the RK stage accumulation, the time-step
// reduction and the conservation sums stay FP64.  Each stage reads the FP64
// state, converts it once to FP32 in shared memory, and adds the FP32 flux
// divergence to the FP64 state in FP64.
#include <algorithm>
#include <new>

#define FSL_CHK_UNIT FSL_CHK_FUSED32
#include "fsl_stage.cuh"
#include "fsl_stage_wide.cuh"

FSL_CHK_EXPORT(fused32)

namespace fsl {

static stage::BF<float> bf32(Ctx &c)
{
    stage::BF<float> b;
    b.x0 = c.bf32.x0; b.xL = c.bf32.xL; b.y0 = c.bf32.y0; b.yH = c.bf32.yH; b.z0 = c.bf32.z0; b.zD = c.bf32.zD;
    return b;
}

void launch_bface32(Ctx &c, const double *cur, const Disturb &d)
{
    stage::launch_bface_t<float>(c, cur, d, bf32(c));
}

template <bool SST>
static int stage32(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant, float *vel)
{
    if (c.p.recon == FSL_RECON_PPM) {
        // PPM: halo 2, a ring of four planes; 16 rows measured fastest at
        // 512x256x256 (11.7 ms per step against 13.4 for 8 rows, two blocks per SM)
        switch (c.stage_tje) {
        case 8: return stage::launch_stage_t<float, 8, 2, true, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
        case 12: return stage::launch_stage_t<float, 12, 1, true, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
        default: return stage::launch_stage_t<float, 16, 1, true, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
        }
    }
    switch (c.stage_tje) {
    case 0: return wide::launch_wide<SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant, vel);
    case 8: return stage::launch_stage_t<float, 8, 2, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    case 12: return stage::launch_stage_t<float, 12, 1, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    default: return stage::launch_stage_t<float, 16, 1, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    }
}

int launch_stage32(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant, float *vel)
{
    // the static Smagorinsky model forms the face viscosity in the kernel
    if (c.p.sgs == FSL_SGS_STATIC) return stage32<true>(c, stage, cur, un, out, courant, vel);
    return stage32<false>(c, stage, cur, un, out, courant, vel);
}

// ---- persistent multi-domain stages ------------------------------------------
struct WidePlan {
    bool sst = false;
    int nblk = 0;
    wide::WideMember *mem = nullptr; // device
    int2 *items = nullptr;           // device
    int *start = nullptr;            // device
    unsigned *bar = nullptr;         // device: count, gen, err
    unsigned limit = 1u << 24;       // barrier polls (64 ns sleeps) before giving up
    int nmem = 0;
};

int wide_plan_build(const std::vector<Ctx *> &members, WidePlan **out, std::string &why)
{
    *out = nullptr;
    if (members.empty()) return FSL_ERR_ARG;
    const bool sst = members[0]->p.sgs == FSL_SGS_STATIC;
    for (Ctx *c : members) {
        if (c->p.precision != FSL_PREC_FP32 || c->p.recon != FSL_RECON_CHARMINMOD || c->stage_tje != 0 ||
            c->p.setup != FSL_SETUP_TEMPORAL || c->p.nStages != 3) {
            why = "members are not all FP32-bulk, reference-scheme, full-lane-tile temporal layers";
            return FSL_ERR_UNSUPPORTED;
        }
        if ((c->p.sgs == FSL_SGS_STATIC) != sst) {
            why = "members mix the static SGS model with others";
            return FSL_ERR_UNSUPPORTED;
        }
        if (!c->fp32_alloc || !c->bf_alloc) {
            why = "a member has not stepped yet";
            return FSL_ERR_ARG;
        }
    }
    const size_t smem = sizeof(wide::Smem<float>);
    const bool attr = sst ? wide::wide_attr<true, true>() : wide::wide_attr<false, true>();
    int per_sm = 0;
    const void *fn = sst ? (const void *)wide::k_wide<true, true> : (const void *)wide::k_wide<false, true>;
    if (!attr || cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, wide::NT, smem) != cudaSuccess ||
        per_sm < 1) {
        why = "persistent stage kernel does not fit on an SM";
        return FSL_ERR_UNSUPPORTED;
    }
    const int sms = members[0]->sms;
    const int nblk = sms * per_sm;
    // the members' own launch splits, balanced over the persistent blocks
    // (longest first, each to the least loaded block)
    std::vector<wide::WideMember> hm;
    struct Item { int m, b; long long cost; };
    std::vector<Item> items;
    for (size_t q = 0; q < members.size(); q++) {
        Ctx &c = *members[q];
        hm.push_back(wide::wide_member(c, c.mu32, bf32(c), c.sms));
        const wide::WideMember &m = hm.back();
        const long long total = (long long)((m.g.D + wide::WK - 1) / wide::WK) * ((m.g.H + wide::WJ - 1) / wide::WJ) * m.g.L;
        for (int b = 0; b < m.nb; b++)
            items.push_back({(int)q, b, total * (b + 1) / m.nb - total * b / m.nb + 2});
    }
    std::vector<int> order(items.size());
    for (size_t q = 0; q < order.size(); q++) order[q] = (int)q;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return items[x].cost > items[y].cost; });
    std::vector<long long> load(nblk, 0);
    std::vector<std::vector<int2>> per(nblk);
    for (int q : order) {
        int best = 0;
        for (int x = 1; x < nblk; x++)
            if (load[x] < load[best]) best = x;
        load[best] += items[q].cost;
        per[best].push_back(make_int2(items[q].m, items[q].b));
    }
    std::vector<int2> flat;
    std::vector<int> start(nblk + 1, 0);
    for (int x = 0; x < nblk; x++) {
        start[x] = (int)flat.size();
        flat.insert(flat.end(), per[x].begin(), per[x].end());
    }
    start[nblk] = (int)flat.size();
    WidePlan *p = new (std::nothrow) WidePlan();
    if (!p) return FSL_ERR_NOMEM;
    p->sst = sst;
    p->nblk = nblk;
    p->nmem = (int)hm.size();
    bool ok = cudaMalloc((void **)&p->mem, hm.size() * sizeof(wide::WideMember)) == cudaSuccess &&
              cudaMalloc((void **)&p->items, std::max<size_t>(1, flat.size()) * sizeof(int2)) == cudaSuccess &&
              cudaMalloc((void **)&p->start, start.size() * sizeof(int)) == cudaSuccess &&
              cudaMalloc((void **)&p->bar, 3 * sizeof(unsigned)) == cudaSuccess;
    ok = ok && cudaMemcpy(p->mem, hm.data(), hm.size() * sizeof(wide::WideMember), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(p->items, flat.data(), flat.size() * sizeof(int2), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(p->start, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(p->bar, 0, 3 * sizeof(unsigned)) == cudaSuccess;
    if (!ok) {
        wide_plan_free(p);
        why = "persistent plan allocation";
        return FSL_ERR_NOMEM;
    }
    *out = p;
    return FSL_OK;
}

void wide_plan_free(WidePlan *p)
{
    if (!p) return;
    cudaFree(p->mem); cudaFree(p->items); cudaFree(p->start); cudaFree(p->bar);
    delete p;
}

int wide_plan_set_limit(WidePlan *p, unsigned polls)
{
    if (!p) return FSL_ERR_ARG;
    p->limit = polls;
    return FSL_OK;
}

// The three stages of every member, one cooperative launch (all blocks
// resident, as the grid barriers between the stages require).
int wide_plan_launch(WidePlan *p, cudaStream_t st)
{
    wide::WideWork w{};
    w.mem = p->mem;
    w.nmem = p->nmem;
    w.items = p->items;
    w.start = p->start;
    w.s_begin = 1;
    w.s_end = 3;
    w.courant = 1;
    w.bar.count = p->bar;
    w.bar.gen = p->bar + 1;
    w.bar.err = reinterpret_cast<int *>(p->bar + 2);
    w.bar.limit = p->limit;
    void *args[] = {&w};
    const void *fn = p->sst ? (const void *)wide::k_wide<true, true> : (const void *)wide::k_wide<false, true>;
    const cudaError_t e =
        cudaLaunchCooperativeKernel(fn, dim3(p->nblk), dim3(wide::NT), args, sizeof(wide::Smem<float>), st);
    return e == cudaSuccess ? FSL_OK : FSL_ERR_CUDA;
}

int wide_plan_check(WidePlan *p, cudaStream_t st)
{
    unsigned h[3] = {0, 0, 0};
    if (cudaMemcpyAsync(h, p->bar, sizeof h, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return FSL_ERR_CUDA;
    if (h[2] == 0) return FSL_OK;
    // a barrier gave up: the step's states are incomplete; re-arm the barrier
    if (cudaMemsetAsync(p->bar, 0, 3 * sizeof(unsigned), st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess)
        return FSL_ERR_CUDA;
    return FSL_ERR_TIMEOUT;
}

} // namespace fsl
