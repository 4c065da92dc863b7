// fsl_fused32.cu -- FP32-bulk instantiation of the fused stage kernel.
//
// Reconstruction, Riemann and viscous fluxes run in FP32 (compiled with
// --use_fast_math: FMA contraction, approximate FP32 division and square
// root); the conserved variables, the RK stage accumulation, the time-step
// reduction and the conservation sums stay FP64.  Each stage reads the FP64
// state, converts it once to FP32 in shared memory, and adds the FP32 flux
// divergence to the FP64 state in FP64.
#include "fsl_stage.cuh"
#include "fsl_stage_wide.cuh"

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
static int stage32(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant)
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
    case 0: return wide::launch_wide<SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    case 8: return stage::launch_stage_t<float, 8, 2, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    case 12: return stage::launch_stage_t<float, 12, 1, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    default: return stage::launch_stage_t<float, 16, 1, false, SST>(c, stage, cur, un, out, c.mu32, bf32(c), courant);
    }
}

int launch_stage32(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant)
{
    // the static Smagorinsky model forms the face viscosity in the kernel
    if (c.p.sgs == FSL_SGS_STATIC) return stage32<true>(c, stage, cur, un, out, courant);
    return stage32<false>(c, stage, cur, un, out, courant);
}

} // namespace fsl
