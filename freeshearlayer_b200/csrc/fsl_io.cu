// fsl_io.cu -- the driver's files: the backup.dat checkpoint (src/finalize.c,
// src/initialize.c:133-158), the probes.dat records (src/probes.c) with their
// Favre average (favre-average-src/layer2_p.c), the latter both as the
// reference's post-processor over a probes file and accumulated on the device.
#include <cstdio>
#include <cstring>
#include <vector>

#include "fsl_internal.h"

using namespace fsl;

namespace {

// The three probe columns of src/probes.c:21-42: i = LEN/2, 3 LEN/4, LEN at
// k = DEP/2 + 1, rows j = 1..HIG of rho and rho u, as rows[station][var][j].
__global__ void k_probe_rows(Grid g, const double *__restrict__ U, double *__restrict__ rows)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.H) return;
    const int k = g.D / 2 + 1;
    const int st[3] = {g.L / 2, 3 * g.L / 4, g.L};
#pragma unroll
    for (int s = 0; s < 3; s++) {
        const long long c = g.idx(st[s], j + 1, k);
        rows[(s * 2 + 0) * g.H + j] = U[c];
        rows[(s * 2 + 1) * g.H + j] = U[g.fstride + c];
    }
}

__global__ void k_probe_accumulate(Grid g, const double *__restrict__ U, double *__restrict__ acc)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= g.H) return;
    const int k = g.D / 2 + 1;
    const int st[3] = {g.L / 2, 3 * g.L / 4, g.L};
#pragma unroll
    for (int s = 0; s < 3; s++) {
        const long long c = g.idx(st[s], j + 1, k);
        acc[(s * 2 + 0) * g.H + j] += U[c];
        acc[(s * 2 + 1) * g.H + j] += U[g.fstride + c];
    }
}

int io_fail(Ctx &c, int code, const char *what)
{
    c.err = what;
    return code;
}

template <typename R> bool write_reals(FILE *f, const double *x, size_t n)
{
    if (sizeof(R) == sizeof(double)) return fwrite(x, sizeof(double), n, f) == n;
    std::vector<R> b(n);
    for (size_t q = 0; q < n; q++) b[q] = (R)x[q];
    return fwrite(b.data(), sizeof(R), n, f) == n;
}

template <typename R> bool read_reals(FILE *f, double *x, size_t n)
{
    if (sizeof(R) == sizeof(double)) return fread(x, sizeof(double), n, f) == n;
    std::vector<R> b(n);
    if (fread(b.data(), sizeof(R), n, f) != n) return false;
    for (size_t q = 0; q < n; q++) x[q] = (double)b[q];
    return true;
}

bool write_real_values(FILE *f, const double *x, size_t n, int real_bytes)
{
    return real_bytes == 4 ? write_reals<float>(f, x, n) : write_reals<double>(f, x, n);
}

bool read_real_values(FILE *f, double *x, size_t n, int real_bytes)
{
    return real_bytes == 4 ? read_reals<float>(f, x, n) : read_reals<double>(f, x, n);
}

int probe_rows(Ctx &c, double *host)
{
    const int H = c.g.H;
    double *d = c.stage_dev; // scratch: 6 HIG <= LEN HIG 5 DEP
    k_probe_rows<<<(H + 127) / 128, 128, 0, c.stream>>>(c.g, c.U, d);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(host, d, 6 * (size_t)H * sizeof(double), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess)
        return io_fail(c, FSL_ERR_CUDA, "probe rows");
    return FSL_OK;
}

} // namespace

extern "C" {

// src/finalize.c:14-35: per (i, j) the DEP values of U1..U5, then deltaT and
// step, in the solver's `real` (real_bytes 4: the shipped float build; 8: FP64).
int fsl_write_backup(fsl_ctx *h, const char *path, int real_bytes)
{
    if (!h || !path || (real_bytes != 4 && real_bytes != 8)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    std::vector<double> st(n);
    int rc = fsl_download_state(h, st.data());
    if (rc) return rc;
    fsl_info info;
    if ((rc = fsl_get_info(h, &info))) return rc;
    FILE *f = fopen(path, "wb");
    if (!f) return io_fail(c, FSL_ERR_IO, "cannot open the backup file to write");
    const double dt = info.deltaT;
    const int step = (int)info.step;
    const bool ok = write_real_values(f, st.data(), n, real_bytes) && write_real_values(f, &dt, 1, real_bytes) &&
                    fwrite(&step, sizeof step, 1, f) == 1;
    if (fclose(f) != 0 || !ok) return io_fail(c, FSL_ERR_IO, "backup write failed");
    return FSL_OK;
}

// src/initialize.c:133-158 reads the fields, skips deltaT (its fread is
// commented out) and so takes `step` from the first bytes of deltaT.  This
// reader takes the file as Finalize() wrote it: fields, deltaT, step.
int fsl_read_backup(fsl_ctx *h, const char *path, int real_bytes)
{
    if (!h || !path || (real_bytes != 4 && real_bytes != 8)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const size_t n = (size_t)c.p.LEN * c.p.HIG * 5 * c.p.DEP;
    FILE *f = fopen(path, "rb");
    if (!f) return io_fail(c, FSL_ERR_IO, "cannot open the backup file to read");
    fseek(f, 0, SEEK_END);
    const long long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size != (long long)((n + 1) * real_bytes + sizeof(int))) {
        fclose(f);
        return io_fail(c, FSL_ERR_IO, "backup file size does not match the grid and real size");
    }
    std::vector<double> st(n);
    double dt = 0;
    int step = 0;
    const bool ok = read_real_values(f, st.data(), n, real_bytes) && read_real_values(f, &dt, 1, real_bytes) &&
                    fread(&step, sizeof step, 1, f) == 1;
    fclose(f);
    if (!ok || step < 0 || !(dt > 0)) return io_fail(c, FSL_ERR_IO, "backup read failed");
    int rc = fsl_upload_state(h, st.data());
    if (rc) return rc;
    return fsl_set_time(h, (unsigned)step, dt);
}

int fsl_probe_rows(fsl_ctx *h, double *rows)
{
    if (!h || !rows) return FSL_ERR_ARG;
    return probe_rows(h->c, rows);
}

// One Probes() record (src/probes.c:13-44) appended to `path`: step, then for
// each station HIG values of rho and HIG values of rho u, in `real`.
int fsl_write_probes(fsl_ctx *h, const char *path, int real_bytes)
{
    if (!h || !path || (real_bytes != 4 && real_bytes != 8)) return FSL_ERR_ARG;
    Ctx &c = h->c;
    std::vector<double> rows(6 * (size_t)c.g.H);
    int rc = probe_rows(c, rows.data());
    if (rc) return rc;
    FILE *f = fopen(path, "ab");
    if (!f) return io_fail(c, FSL_ERR_IO, "cannot open the probes file");
    const int step = (int)c.step;
    const bool ok = fwrite(&step, sizeof step, 1, f) == 1 && write_real_values(f, rows.data(), rows.size(), real_bytes);
    if (fclose(f) != 0 || !ok) return io_fail(c, FSL_ERR_IO, "probes write failed");
    return FSL_OK;
}

// Device-side sums of the probe columns (the Favre post-processor's R and
// rho U sums, favre-average-src/layer2_p.c:59-104, without a probes file).
int fsl_favre_reset(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    if (!c.favre) {
        if (cudaMalloc((void **)&c.favre, 6 * (size_t)c.g.H * sizeof(double)) != cudaSuccess)
            return io_fail(c, FSL_ERR_NOMEM, "favre accumulators");
        c.bytes += 6 * (size_t)c.g.H * sizeof(double);
    }
    if (cudaMemsetAsync(c.favre, 0, 6 * (size_t)c.g.H * sizeof(double), c.stream) != cudaSuccess)
        return io_fail(c, FSL_ERR_CUDA, "favre reset");
    c.favre_count = 0;
    return FSL_OK;
}

int fsl_favre_accumulate(fsl_ctx *h)
{
    if (!h) return FSL_ERR_ARG;
    Ctx &c = h->c;
    int rc;
    if (!c.favre && (rc = fsl_favre_reset(h))) return rc;
    k_probe_accumulate<<<(c.g.H + 127) / 128, 128, 0, c.stream>>>(c.g, c.U, c.favre);
    if (cudaGetLastError() != cudaSuccess) return io_fail(c, FSL_ERR_CUDA, "favre accumulate");
    c.favre_count++;
    return FSL_OK;
}

// Favre-averaged streamwise velocity per station and row, sum(rho u) / sum(rho)
// (favre-average-src/layer2_p.c:106-112), as u[station][j]; *count = records.
int fsl_favre_read(fsl_ctx *h, double *u, int *count)
{
    if (!h || !u) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const int H = c.g.H;
    std::vector<double> acc(6 * (size_t)H, 0.0);
    if (c.favre &&
        (cudaMemcpyAsync(acc.data(), c.favre, acc.size() * sizeof(double), cudaMemcpyDeviceToHost, c.stream) !=
             cudaSuccess ||
         cudaStreamSynchronize(c.stream) != cudaSuccess))
        return io_fail(c, FSL_ERR_CUDA, "favre read");
    for (int s = 0; s < 3; s++)
        for (int j = 0; j < H; j++) u[s * H + j] = acc[(s * 2 + 1) * H + j] / acc[(s * 2) * H + j];
    if (count) *count = c.favre_count;
    return FSL_OK;
}

// The reference's post-processor over a probes file (favre-average-src/
// layer2_p.c:59-112): records with step_start <= step <= step_end are summed
// per station and row; it stops at the first record past step_end or at the
// end of the file (the reference loops on a failed read there).  Host only.
int fsl_favre_from_probes(const char *path, int HIG, int real_bytes, int step_start, int step_end, double *u,
                          int *records)
{
    if (!path || HIG < 1 || !u || (real_bytes != 4 && real_bytes != 8)) return FSL_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return FSL_ERR_IO;
    std::vector<double> R(3 * (size_t)HIG, 0.0), RU(3 * (size_t)HIG, 0.0), rec(6 * (size_t)HIG);
    int n = 0, step = 0;
    for (;;) {
        if (fread(&step, sizeof step, 1, f) != 1) break;
        if (step > step_end) break;
        if (!read_real_values(f, rec.data(), rec.size(), real_bytes)) break;
        if (step < step_start) continue;
        for (int s = 0; s < 3; s++)
            for (int j = 0; j < HIG; j++) {
                R[s * HIG + j] += rec[(s * 2) * HIG + j];
                RU[s * HIG + j] += rec[(s * 2 + 1) * HIG + j];
            }
        n++;
    }
    fclose(f);
    for (size_t q = 0; q < R.size(); q++) u[q] = RU[q] / R[q];
    if (records) *records = n;
    return FSL_OK;
}

} // extern "C"
