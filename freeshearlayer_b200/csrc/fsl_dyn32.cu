// fsl_dyn32.cu -- the dynamic Smagorinsky procedure in FP32 for the FP32-bulk
// path (filters, Leonard stress, strain rates and coefficient in FP32 from
// the FP64 state; mu_SGS written as the FP32 field the stage kernel reads).
// The scratch fields are the FP64 path's, each holding `fstride` floats.
#include <algorithm>

#include "fsl_dyn.cuh"

namespace fsl {

void launch_dynsmag32(Ctx &c, const double *U, float *cd)
{
    const DynScratch &s = c.dyn;
    const dyn::Scratch<float> sc{reinterpret_cast<float *>(s.vel), reinterpret_cast<float *>(s.t1),
                                 reinterpret_cast<float *>(s.t2),  reinterpret_cast<float *>(s.A),
                                 reinterpret_cast<float *>(s.Lst), reinterpret_cast<float *>(s.B),
                                 reinterpret_cast<float *>(s.S)};
    prof_begin(c, FSL_K_SGS);
    dyn::sequence<float>(c.g, c.k, sc, U, c.mu32, cd, c.stream);
    prof_end(c, FSL_K_SGS, 9);
}

} // namespace fsl
