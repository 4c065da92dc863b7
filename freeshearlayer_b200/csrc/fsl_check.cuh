// fsl_check.cuh -- debug bounds checks of global-memory indices.
//
// Built with -DFSL_BOUNDS_CHECK=1 (`make -C freeshearlayer_b200 checked`,
// libfsl_gpu_checked.so), every index wrapped in FSL_CELL or FSL_FACE is
// tested against the extent of the array it indexes before the access: a
// cell index against one field of the padded box ([0, fstride); the field
// offset q * fstride is added outside the check), a face index against one
// field of a boundary-face array.  The first offending access records its
// translation unit, source line, index and extent in a device word of that
// unit, every offending access counts, and the access is redirected to
// element 0 so it cannot leave the allocation.  fsl_debug_bounds reads the
// records.  In the product build the macros are the bare index.
#pragma once

#include <cuda_runtime.h>

namespace fsl {
namespace chk {

struct Record {
    unsigned long long hits; // offending accesses since the last clear
    int unit, line;          // of the first one
    long long index, extent;
};

// The checks on an explicit record, compiled for host and device: the device
// counts with an atomic, the host (single-threaded: the CPU test of this
// logic) with a plain increment.
__host__ __device__ inline void record_into(Record *r, long long i, long long n, int unit, int line)
{
#ifdef __CUDA_ARCH__
    const unsigned long long before = atomicAdd(&r->hits, 1ull);
#else
    const unsigned long long before = r->hits++;
#endif
    if (before == 0ull) {
        r->unit = unit;
        r->line = line;
        r->index = i;
        r->extent = n;
    }
}

// i itself when 0 <= i < n; otherwise recorded, and 0
__host__ __device__ inline long long at_into(Record *r, long long i, long long n, int unit, int line)
{
    if ((unsigned long long)i < (unsigned long long)n) return i;
    record_into(r, i, n, unit, line);
    return 0;
}

// the stencil c + lo .. c + hi (lo <= 0 <= hi) inside [0, n); otherwise the
// offending extreme is recorded
__host__ __device__ inline bool span_into(Record *r, long long c, long long lo, long long hi, long long n, int unit,
                                          int line)
{
    if (c + lo >= 0 && c + hi < n) return true;
    record_into(r, c + lo < 0 ? c + lo : c + hi, n, unit, line);
    return false;
}

#if FSL_BOUNDS_CHECK
// one record per translation unit (no relocatable device code needed)
static __device__ Record g_rec;

__device__ __forceinline__ long long at(long long i, long long n, int unit, int line)
{
    return at_into(&g_rec, i, n, unit, line);
}

__device__ __forceinline__ bool span(long long c, long long lo, long long hi, long long n, int unit, int line)
{
    return span_into(&g_rec, c, lo, hi, n, unit, line);
}

// this unit's record, read (and with clear, reset) from the host
static inline int read_unit(Record *out, bool clear)
{
    if (cudaMemcpyFromSymbol(out, g_rec, sizeof(Record)) != cudaSuccess) return -1;
    if (clear) {
        const Record z{};
        if (cudaMemcpyToSymbol(g_rec, &z, sizeof(Record)) != cudaSuccess) return -1;
    }
    return 0;
}
#endif

} // namespace chk
} // namespace fsl

namespace fsl {
// the units' record readers (-1 when built without checks)
int chk_read_fused(chk::Record *out, bool clear);
int chk_read_fused32(chk::Record *out, bool clear);
int chk_read_mlp(chk::Record *out, bool clear);
int chk_read_phase(chk::Record *out, bool clear);
int chk_read_dyn32(chk::Record *out, bool clear);
int chk_read_io(chk::Record *out, bool clear);
} // namespace fsl

// Translation-unit ids of the records (FSL_CHK_UNIT must be defined before
// this header in every unit that checks).
#define FSL_CHK_FUSED 1   // fsl_fused.cu: FP64 ring-tile stage kernels
#define FSL_CHK_FUSED32 2 // fsl_fused32.cu: FP32 ring-tile and full-lane stage kernels, ensembles
#define FSL_CHK_MLP 3     // fsl_mlp.cu: closure features and inference
#define FSL_CHK_PHASE 4   // fsl_phase.cu: per-phase kernels, state transfers, reductions, FP64 dynamic procedure
#define FSL_CHK_DYN32 5   // fsl_dyn32.cu: FP32 dynamic procedure
#define FSL_CHK_IO 6      // fsl_io.cu: probes and Tecplot fields

#if FSL_BOUNDS_CHECK
#define FSL_CELL(c, fs) (::fsl::chk::at((c), (fs), FSL_CHK_UNIT, __LINE__))
#define FSL_FACE(f, n) (::fsl::chk::at((f), (n), FSL_CHK_UNIT, __LINE__))
// a stencil's extremes: true when inside (a kernel without block barriers
// skips the cell otherwise); always true in the product build
#define FSL_SPAN(c, lo, hi, n) (::fsl::chk::span((c), (lo), (hi), (n), FSL_CHK_UNIT, __LINE__))
// the host reader of this unit's record: int fsl_chk_read_<name>(Record*, bool)
#define FSL_CHK_EXPORT(name)                                                                                          \
    namespace fsl {                                                                                                   \
    int chk_read_##name(chk::Record *out, bool clear) { return chk::read_unit(out, clear); }                         \
    }
#else
#define FSL_CELL(c, fs) (c)
#define FSL_FACE(f, n) (f)
#define FSL_SPAN(c, lo, hi, n) true
#define FSL_CHK_EXPORT(name)                                                                                          \
    namespace fsl {                                                                                                   \
    int chk_read_##name(chk::Record *, bool) { return -1; }                                                           \
    }
#endif
