// fsl_fused.cu -- FP64 instantiation of the fused stage kernel (the plain
// method).  Compiled with --fmad=false: every value is formed with the
// reference's expressions and rounds exactly like the reference's serial code.
#define FSL_CHK_UNIT FSL_CHK_FUSED
#include "fsl_stage.cuh"

FSL_CHK_EXPORT(fused)

namespace fsl {

static stage::BF<double> bf64(Ctx &c)
{
    stage::BF<double> b;
    b.x0 = c.bf.x0; b.xL = c.bf.xL; b.y0 = c.bf.y0; b.yH = c.bf.yH; b.z0 = c.bf.z0; b.zD = c.bf.zD;
    return b;
}

void launch_bface(Ctx &c, const double *cur, const Disturb &d)
{
    stage::launch_bface_t<double>(c, cur, d, bf64(c));
}

template <bool SST>
static int stage64(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant)
{
    // PPM: halo 2, a ring of four planes.  A 16-row FP64 tile would need more
    // than the 227 KB of shared memory a block may have; 12 rows measured
    // fastest at 512x256x256 (54 ms per step against 69 for 8), so 16 runs as 12
    if (c.p.recon == FSL_RECON_PPM) {
        if (c.stage_tje == 8)
            return stage::launch_stage_t<double, 8, 1, true, SST>(c, stage, cur, un, out, c.mu, bf64(c), courant);
        return stage::launch_stage_t<double, 12, 1, true, SST>(c, stage, cur, un, out, c.mu, bf64(c), courant);
    }
    switch (c.stage_tje) {
    case 8: return stage::launch_stage_t<double, 8, 1, false, SST>(c, stage, cur, un, out, c.mu, bf64(c), courant);
    case 12: return stage::launch_stage_t<double, 12, 1, false, SST>(c, stage, cur, un, out, c.mu, bf64(c), courant);
    default: return stage::launch_stage_t<double, 16, 1, false, SST>(c, stage, cur, un, out, c.mu, bf64(c), courant);
    }
}

int launch_stage(Ctx &c, int stage, const double *cur, const double *un, double *out, bool courant)
{
    // the static Smagorinsky model forms the face viscosity in the kernel
    if (c.p.sgs == FSL_SGS_STATIC) return stage64<true>(c, stage, cur, un, out, courant);
    return stage64<false>(c, stage, cur, un, out, courant);
}

} // namespace fsl
