// fsl_dyn32.cu -- the dynamic Smagorinsky procedure in FP32 for the FP32-bulk
// path (filters, Leonard stress, strain rates and coefficient in FP32 from
// the FP64 state; mu_SGS written as the FP32 field the stage kernel reads).
// Its scratch fields are FP32 buffers of its own (DynScratch32).
#include <algorithm>

#define FSL_CHK_UNIT FSL_CHK_DYN32
#include "fsl_dyn.cuh"

FSL_CHK_EXPORT(dyn32)

namespace fsl {

void launch_dynsmag32(Ctx &c, const double *U, float *cd)
{
    const DynScratch32 &s = c.dyn32;
    const dyn::Scratch3<float> sc{s.vel, s.F, s.A, s.S};
    prof_begin(c, FSL_K_SGS);
    dyn::sequence_fused<float>(c.g, c.k, sc, U, c.mu32, cd, c.stream);
    prof_end(c, FSL_K_SGS, 4);
}

} // namespace fsl
