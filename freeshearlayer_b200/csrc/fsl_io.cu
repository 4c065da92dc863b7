// fsl_io.cu -- the driver's files: the backup.dat checkpoint (src/finalize.c,
// src/initialize.c:133-158), the probes.dat records (src/probes.c) with their
// Favre average (favre-average-src/layer2_p.c), the latter both as the
// reference's post-processor over a probes file and accumulated on the device.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#define FSL_CHK_UNIT FSL_CHK_IO
#include "fsl_check.cuh"
#include "fsl_internal.h"

FSL_CHK_EXPORT(io)

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
        const long long c = FSL_CELL(g.idx(st[s], j + 1, k), g.fstride);
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
        const long long c = FSL_CELL(g.idx(st[s], j + 1, k), g.fstride);
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
    ApiRange range_("fsl_write_backup");
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

// The reference post-processor's whole job on a float probes file
// (favre-average-src/layer2_p.c:30-146): per station, the records with
// step_start <= step <= step_end summed in float in file order, u~ = sum(rho
// u) / sum(rho) in float, and the three profile files probe1.dat ..
// probe3.dat in its text format.  Unlike the reference's reader, which
// re-adds its last record for ever when the file ends before a step beyond
// step_end, reading stops at the end of the file.
int fsl_favre_profiles(const char *path, int HIG, int step_start, int step_end, const char *dir, int *records)
{
    if (!path || HIG < 1 || !dir) return FSL_ERR_ARG;
    FILE *f = fopen(path, "rb");
    if (!f) return FSL_ERR_IO;
    std::vector<float> R(3 * (size_t)HIG, 0.f), RU(3 * (size_t)HIG, 0.f), pr(HIG), pu(HIG);
    unsigned step = 0;
    int n = 0;
    for (;;) {
        if (fread(&step, sizeof step, 1, f) != 1) break;
        if (step > (unsigned)step_end) break;
        bool ok = true;
        for (int st = 0; st < 3 && ok; st++) {
            ok = fread(pr.data(), sizeof(float) * HIG, 1, f) == 1 && fread(pu.data(), sizeof(float) * HIG, 1, f) == 1;
            if (!ok || step < (unsigned)step_start) continue;
            for (int j = 0; j < HIG; j++) {
                R[st * HIG + j] += pr[j];
                RU[st * HIG + j] += pu[j];
            }
        }
        if (!ok) break;
        if (step >= (unsigned)step_start) n++;
    }
    fclose(f);
    for (size_t q = 0; q < RU.size(); q++) RU[q] /= R[q];
    for (int st = 0; st < 3; st++) {
        const std::string name = std::string(dir) + "/probe" + std::to_string(st + 1) + ".dat";
        FILE *o = fopen(name.c_str(), "w");
        if (!o) return FSL_ERR_IO;
        fprintf(o, "%d\n1\n", HIG + 2);
        fprintf(o, "%f %3.2f \n", -0.00001, 0.);
        for (int j = 0; j < HIG; j++) fprintf(o, "%d %3.2f \n", j, RU[st * HIG + j]);
        fprintf(o, "%f %3.2f \n", HIG - 1 + 0.00001, 210.);
        fclose(o);
    }
    if (records) *records = n;
    return FSL_OK;
}

} // extern "C"

// ---- Tecplot frames (src/output.c) -------------------------------------------
namespace {

// Output()'s 12 values per interior cell in its arithmetic (FP64, compiled
// without contraction), written in its loop order: k, then j, then i fastest.
__global__ void k_output_fields(Grid g, Consts kc, double Cs, const double *__restrict__ Ub, double *__restrict__ out)
{
    const long long n = (long long)g.L * g.H * g.D;
    const long long fs = g.fstride;
    const double *U1 = Ub, *U2 = Ub + fs, *U3 = Ub + 2 * fs, *U4 = Ub + 3 * fs, *U5 = Ub + 4 * fs;
    const double CsDD = Cs * kc.DD;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.L) + 1;
        const long long r = t / g.L;
        const int j = (int)(r % g.H) + 1, k = (int)(r / g.H) + 1;
        const long long c = g.idx(i, j, k), xi = g.pi, yj = g.pk;
        if (!FSL_SPAN(c, -xi, xi, fs)) continue; // the strain stencil's extremes
        double *q = out + 12 * t;
        q[0] = (i - 1) * kc.deltaX + 0.5 * kc.deltaX;
        q[1] = (j - 1) * kc.deltaY + 0.5 * kc.deltaY;
        q[2] = (k - 1) * kc.deltaZ + 0.5 * kc.deltaZ;
        const double R = U1[c], Uu = U2[c] / R, V = U3[c] / R, W = U4[c] / R;
        const double P = (U5[c] - 0.5 * R * (Uu * Uu + V * V + W * W)) * 0.4;
        const double T = P / (287.10 * R);
        const double du_dx = (U2[c + xi] / U1[c + xi] - U2[c - xi] / U1[c - xi]) * kc.r2dx;
        const double du_dy = (U2[c + yj] / U1[c + yj] - U2[c - yj] / U1[c - yj]) * kc.r2dy;
        const double du_dz = (U2[c + 1] / U1[c + 1] - U2[c - 1] / U1[c - 1]) * kc.r2dz;
        const double dv_dx = (U3[c + xi] / U1[c + xi] - U3[c - xi] / U1[c - xi]) * kc.r2dx;
        const double dv_dy = (U3[c + yj] / U1[c + yj] - U3[c - yj] / U1[c - yj]) * kc.r2dy;
        const double dv_dz = (U3[c + 1] / U1[c + 1] - U3[c - 1] / U1[c - 1]) * kc.r2dz;
        const double dw_dx = (U4[c + xi] / U1[c + xi] - U4[c - xi] / U1[c - xi]) * kc.r2dx;
        const double dw_dy = (U4[c + yj] / U1[c + yj] - U4[c - yj] / U1[c - yj]) * kc.r2dy;
        const double dw_dz = (U4[c + 1] / U1[c + 1] - U4[c - 1] / U1[c - 1]) * kc.r2dz;
        const double ox = dw_dy - dv_dz, oy = du_dz - dw_dx, oz = dv_dx - du_dy;
        const double Om = sqrt(ox * ox + oy * oy + oz * oz);
        const double S12 = 0.5 * (du_dy + dv_dx), S13 = 0.5 * (du_dz + dw_dx), S23 = 0.5 * (dv_dz + dw_dy);
        const double St =
            sqrt(2 * (du_dx * du_dx + dv_dy * dv_dy + dw_dz * dw_dz + 2 * (S12 * S12 + S13 * S13 + S23 * S23)));
        q[3] = R; q[4] = Uu; q[5] = V; q[6] = W; q[7] = P; q[8] = T;
        q[9] = Om;
        q[10] = 0.5 * (Om * Om - St * St);
        q[11] = R * CsDD * St / kc.mu_L;
    }
}

} // namespace

extern "C" {

int fsl_output_fields(fsl_ctx *h, double *out)
{
    if (!h || !out) return FSL_ERR_ARG;
    Ctx &c = h->c;
    const size_t n = (size_t)c.g.L * c.g.H * c.g.D;
    double *d = nullptr;
    if (cudaMalloc((void **)&d, 12 * n * sizeof(double)) != cudaSuccess)
        return io_fail(c, FSL_ERR_NOMEM, "output fields");
    k_output_fields<<<148 * 8, 256, 0, c.stream>>>(c.g, c.k, c.p.Cs, c.U, d);
    const bool ok = cudaGetLastError() == cudaSuccess &&
                    cudaMemcpyAsync(out, d, 12 * n * sizeof(double), cudaMemcpyDeviceToHost, c.stream) == cudaSuccess &&
                    cudaStreamSynchronize(c.stream) == cudaSuccess;
    cudaFree(d);
    return ok ? FSL_OK : io_fail(c, FSL_ERR_CUDA, "output fields");
}

// The ASCII Tecplot file of src/output.c:66-139 from the 12 values per cell.
int fsl_tecplot_write(const char *path, int LEN, int HIG, int DEP, const double *fields)
{
    if (!path || !fields || LEN < 1 || HIG < 1 || DEP < 1) return FSL_ERR_ARG;
    FILE *f = fopen(path, "w");
    if (!f) return FSL_ERR_IO;
    fprintf(f, "title     = \" 3-D compressible case \"\n");
    fprintf(f, "variables = \" x \"\n");
    fprintf(f, "\"y\"\n\"z\"\n\"rho\"\n\"u\"\n\"v\"\n\"w\"\n\"p\"\n\"T\"\n");
    fprintf(f, "\"Vort. mag.\"\n\"Q-criteria.\"\n\"muSgs-mu-ratio\"\n");
    fprintf(f, "zone t=\" \"\n");
    fprintf(f, "i=%d, j=%d, k=%d, f=point\n", LEN, HIG, DEP);
    const size_t n = (size_t)LEN * HIG * DEP;
    for (size_t t = 0; t < n; t++) {
        const double *q = fields + 12 * t;
        fprintf(f, "%g %g %g %g %g %g %g %g %g %g %g %g\n", q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], q[8],
                q[9], q[10], q[11]);
    }
    return fclose(f) == 0 ? FSL_OK : FSL_ERR_IO;
}

// Output(): "<path>" written from the current U^n (call it after fsl_step,
// where the reference calls Output() after the stages).
int fsl_write_tecplot(fsl_ctx *h, const char *path)
{
    if (!h || !path) return FSL_ERR_ARG;
    Ctx &c = h->c;
    std::vector<double> q(12 * (size_t)c.g.L * c.g.H * c.g.D);
    int rc = fsl_output_fields(h, q.data());
    if (rc) return rc;
    rc = fsl_tecplot_write(path, c.g.L, c.g.H, c.g.D, q.data());
    return rc ? io_fail(c, rc, "tecplot write failed") : FSL_OK;
}

} // extern "C"
