/*
 * ref_static.h -- second forced include (after ref_patch.h) used ONLY to
 * compile the reference's src/fluxes.c a second time, in place, into the test
 * oracle oracle/_ref/libfslref.so as Fluxes_static().  Test infrastructure,
 * never linked by the product.
 *
 * The reference selects its SGS model with a hardcoded macro: src/def.h:47
 * sets DynamicSmagorinskySGS 1 (the dynamic procedure), src-par/def.h:47 sets
 * it 0 (the static Smagorinsky branch of src/fluxes.c:193-205, :362-374,
 * :533-545).  def.h is guarded by DEF_H, so including it here first and then
 * redefining the macro makes fluxes.c compile its static branch without any
 * edit to the reference tree.
 */
#include "def.h"
#undef DynamicSmagorinskySGS
#define DynamicSmagorinskySGS 0
