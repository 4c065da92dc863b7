// fsl_phase.cu -- one kernel per reference phase of the explicit step (FP64).
//
// These are the unfused path behind the per-phase C-ABI entry points
// (fsl_ghost_bc, fsl_reconstruct, ...).  They keep the reference's data flow
// (face-state arrays between reconstruction and fluxes) so each phase can be
// checked on its own against the CPU oracle.  Compiled with --fmad=false:
// results equal the reference's serial FP64 code bit for bit.
#include <algorithm>

#define FSL_CHK_UNIT FSL_CHK_PHASE
#include "fsl_check.cuh"
#include "fsl_dyn.cuh"
#include "fsl_internal.h"
#include "fsl_phys.cuh"

FSL_CHK_EXPORT(phase)

namespace fsl {

namespace {

__device__ __forceinline__ long long ixf(int L, int H, int D, int i, int j, int k)
{
    return FSL_FACE(((long long)i * H + j) * D + k, (long long)(L + 1) * H * D);
}
__device__ __forceinline__ long long iyf(int L, int H, int D, int i, int j, int k)
{
    return FSL_FACE(((long long)i * (H + 1) + j) * D + k, (long long)L * (H + 1) * D);
}
__device__ __forceinline__ long long izf(int L, int H, int D, int i, int j, int k)
{
    return FSL_FACE(((long long)i * H + j) * (D + 1) + k, (long long)L * H * (D + 1));
}

// ---------------------------------------------------------------------------
// A1 ghost cells (src/boundCondInGhostCells.c:10-96).  The reference fills x,
// then z over all i, then y over all i and k; every ghost value is therefore a
// composition of copies of one interior cell (or of the inflow profile).  Each
// thread evaluates that composition for one ghost cell, so all ghost cells are
// written in one pass with the reference's values, edges and corners included.
// ---------------------------------------------------------------------------
__global__ void k_ghost(Grid g, int setup, double *__restrict__ u)
{
    const int L = g.L, H = g.H, D = g.D;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nx = 2LL * (H + 2) * (D + 2), ny = 2LL * L * (D + 2), nz = 2LL * L * H;
    int i, j, k;
    if (t < nx) {
        long long a = (long long)(H + 2) * (D + 2);
        i = (t / a) ? L + 1 : 0;
        long long r = t % a;
        j = (int)(r / (D + 2));
        k = (int)(r % (D + 2));
    } else if ((t -= nx) < ny) {
        long long a = (long long)L * (D + 2);
        j = (t / a) ? H + 1 : 0;
        long long r = t % a;
        i = 1 + (int)(r / (D + 2));
        k = (int)(r % (D + 2));
    } else if ((t -= ny) < nz) {
        long long a = (long long)L * H;
        k = (t / a) ? D + 1 : 0;
        long long r = t % a;
        i = 1 + (int)(r / H);
        j = 1 + (int)(r % H);
    } else {
        return;
    }
    const bool spatial = (setup == FSL_SETUP_SPATIAL);
    bool flip = false;
    int jj = j, kk = k;
    if (j == 0) { jj = 1; flip = spatial; }
    else if (j == H + 1) { jj = H; flip = spatial; }
    if (k == 0) kk = D;
    else if (k == D + 1) kk = 1;
    double v[5];
    const long long fs = g.fstride;
    typedef Kc<double> kc;
    if (i == 0 && spatial) {
        // inflow step profile, :17-40
        const double P = 100000., R = 1.0;
        const double U = (jj <= H / 2) ? 76.4 : 200;
        v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.;
        v[4] = P / kc::K_1 + 0.5 * R * (U * U);
    } else {
        int si = i;
        if (i == 0) si = L;               // temporal: periodic x
        else if (i == L + 1) si = spatial ? L : 1;
        long long s = FSL_CELL(g.idx(si, jj, kk), fs);
#pragma unroll
        for (int q = 0; q < 5; q++) v[q] = u[q * fs + s];
        if (i == L + 1 && spatial) {
            // outflow, :44-52: momenta copied, E rebuilt at P = 1e5
            const double P = 100000.;
            v[4] = P / kc::K_1 + 0.5 * (v[1] * v[1] + v[2] * v[2] + v[3] * v[3]) / v[0];
        }
    }
    if (flip) v[2] = -v[2];
    long long d = FSL_CELL(g.idx(i, j, k), fs);
#pragma unroll
    for (int q = 0; q < 5; q++) u[q * fs + d] = v[q];
}

// ---------------------------------------------------------------------------
// A2 reconstruction (src/reconstruction.c:26-345): one thread per interior
// cell, all three sweeps, six face states written to the face arrays.  With
// PPM, a sweep whose four neighbours exist (the cell is not next to the
// domain boundary in that direction) uses ppm_* instead.
// ---------------------------------------------------------------------------
template <bool PPM>
__global__ void __launch_bounds__(128) k_recon(Grid g, const double *__restrict__ u, Faces f)
{
    const int L = g.L, H = g.H, D = g.D;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > D || j > H) return;
    const long long fs = g.fstride;
    const long long c0 = g.idx(i, j, k);
    if (!FSL_SPAN(c0, -g.pi, g.pi, fs)) return; // the one-neighbour stencil in x, the widest
    CellC<double> c;
#pragma unroll
    for (int q = 0; q < 5; q++) c.u[q] = u[q * fs + c0];
    cell_consts(c);
    double fw[5], bw[5], hi[5], lo[5];
    // x
    {
        const long long a = c0 + g.pi, b = c0 - g.pi;
#pragma unroll
        for (int q = 0; q < 5; q++) { fw[q] = u[q * fs + a]; bw[q] = u[q * fs + b]; }
        if (PPM && i >= 2 && i <= L - 1) {
            double m2[5], p2[5];
#pragma unroll
            for (int q = 0; q < 5; q++) { p2[q] = u[q * fs + a + g.pi]; m2[q] = u[q * fs + b - g.pi]; }
            ppm_x(c, m2, bw, fw, p2, hi, lo);
        } else {
            recon_x(c, fw, bw, hi, lo);
        }
        const long long fh = ixf(L, H, D, i, j - 1, k - 1), fl = ixf(L, H, D, i - 1, j - 1, k - 1);
#pragma unroll
        for (int q = 0; q < 5; q++) { f.x[0][q][fh] = hi[q]; f.x[1][q][fl] = lo[q]; }
    }
    // y: (rho, rho v, rho w, rho u, E)
    {
        const long long a = c0 + g.pk, b = c0 - g.pk;
        const int perm[5] = {0, 2, 3, 1, 4};
#pragma unroll
        for (int q = 0; q < 5; q++) { fw[q] = u[perm[q] * fs + a]; bw[q] = u[perm[q] * fs + b]; }
        if (PPM && j >= 2 && j <= H - 1) {
            double m2[5], p2[5];
#pragma unroll
            for (int q = 0; q < 5; q++) { p2[q] = u[perm[q] * fs + a + g.pk]; m2[q] = u[perm[q] * fs + b - g.pk]; }
            ppm_y(c, m2, bw, fw, p2, hi, lo);
        } else {
            recon_y(c, fw, bw, hi, lo);
        }
        const long long fh = iyf(L, H, D, i - 1, j, k - 1), fl = iyf(L, H, D, i - 1, j - 1, k - 1);
#pragma unroll
        for (int q = 0; q < 5; q++) { f.y[0][q][fh] = hi[q]; f.y[1][q][fl] = lo[q]; }
    }
    // z: (rho, rho w, rho u, rho v, E)
    {
        const long long a = c0 + 1, b = c0 - 1;
        const int perm[5] = {0, 3, 1, 2, 4};
#pragma unroll
        for (int q = 0; q < 5; q++) { fw[q] = u[perm[q] * fs + a]; bw[q] = u[perm[q] * fs + b]; }
        if (PPM && k >= 2 && k <= D - 1) {
            double m2[5], p2[5];
#pragma unroll
            for (int q = 0; q < 5; q++) { p2[q] = u[perm[q] * fs + a + 1]; m2[q] = u[perm[q] * fs + b - 1]; }
            ppm_z(c, m2, bw, fw, p2, hi, lo);
        } else {
            recon_z(c, fw, bw, hi, lo);
        }
        const long long fh = izf(L, H, D, i - 1, j - 1, k), fl = izf(L, H, D, i - 1, j - 1, k - 1);
#pragma unroll
        for (int q = 0; q < 5; q++) { f.z[0][q][fh] = hi[q]; f.z[1][q][fl] = lo[q]; }
    }
}

// ---------------------------------------------------------------------------
// A3 boundary face states (src/bounCondOnInterfaces.c:11-110).
// ---------------------------------------------------------------------------
__global__ void k_ifbc(Grid g, int setup, int BL_HIG, Disturb d, Faces f)
{
    const int L = g.L, H = g.H, D = g.D;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nx = (long long)H * D, ny = (long long)L * D, nz = (long long)L * H;
    const bool spatial = (setup == FSL_SETUP_SPATIAL);
    typedef Kc<double> kc;
    if (t < nx) {
        const int j = (int)(t / D), k = (int)(t % D);
        const long long f0 = ixf(L, H, D, 0, j, k), fL = ixf(L, H, D, L, j, k);
        if (spatial) {
            const double P = 100000., R = 1.0;
            double U, V = 0., W = 0.;
            double v[5];
            if (j < H / 2) { // :17-29
                U = 76.4;
                v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.; v[4] = P / kc::K_1 + 0.5 * R * (U * U);
            } else if (j < H / 2 + BL_HIG) { // :31-49
                const unsigned ku = (unsigned)k;
                bool dist;
                if (d.k_max > d.k_min) dist = (ku >= d.k_min && ku < d.k_max);
                else dist = !(ku >= d.k_max && ku < d.k_min);
                if (dist) { U = 200. + d.Ud; V = d.Vd; W = d.Wd; }
                else { U = 200.; V = W = 0.; }
                v[0] = R; v[1] = R * U; v[2] = R * V; v[3] = R * W;
                v[4] = P / kc::K_1 + 0.5 * R * (U * U + V * V + W * W);
            } else { // :51-60
                U = 200.;
                v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.; v[4] = P / kc::K_1 + 0.5 * R * (U * U);
            }
#pragma unroll
            for (int q = 0; q < 5; q++) f.x[0][q][f0] = v[q];
            // :62-71 outflow
            const double r = f.x[0][0][fL], mu_ = f.x[0][1][fL], mv = f.x[0][2][fL], mw = f.x[0][3][fL];
            f.x[1][0][fL] = r; f.x[1][1][fL] = mu_; f.x[1][2][fL] = mv; f.x[1][3][fL] = mw;
            f.x[1][4][fL] = P / kc::K_1 + 0.5 * (mu_ * mu_ + mv * mv + mw * mw) / r;
        } else {
#pragma unroll
            for (int q = 0; q < 5; q++) {
                f.x[0][q][f0] = f.x[0][q][fL];
                f.x[1][q][fL] = f.x[1][q][f0];
            }
        }
    } else if ((t -= nx) < ny) { // :75-90
        const int i = (int)(t / D), k = (int)(t % D);
        const long long f0 = iyf(L, H, D, i, 0, k), fH = iyf(L, H, D, i, H, k);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            if (q == 2 && spatial) {
                f.y[0][q][f0] = -f.y[1][q][f0];
                f.y[1][q][fH] = -f.y[0][q][fH];
            } else {
                f.y[0][q][f0] = f.y[1][q][f0];
                f.y[1][q][fH] = f.y[0][q][fH];
            }
        }
    } else if ((t -= ny) < nz) { // :94-109
        const int i = (int)(t / H), j = (int)(t % H);
        const long long f0 = izf(L, H, D, i, j, 0), fD = izf(L, H, D, i, j, D);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            f.z[0][q][f0] = f.z[0][q][fD];
            f.z[1][q][fD] = f.z[1][q][f0];
        }
    }
}

// ---------------------------------------------------------------------------
// A4 fluxes (src/fluxes.c:57-571): one thread per face of direction N.
// The flux overwrites the minus-side state array, as in the reference.
// ---------------------------------------------------------------------------
// sgs: FSL_SGS_STATIC forms the face viscosity from the face gradients and
// the two cells' densities (src/fluxes.c:193-205, :362-374, :533-545),
// FSL_SGS_NONE uses zero, any other mode the mu_SGS field.
template <int N>
__global__ void __launch_bounds__(128) k_flux(Grid g, Consts kc, const double *__restrict__ u,
                                              const double *__restrict__ mu, Faces f, int sgs)
{
    const int L = g.L, H = g.H, D = g.D;
    const int na = L + (N == 1), nb = H + (N == 2), nc = D + (N == 3);
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y * blockDim.y + threadIdx.y;
    const int a = blockIdx.z;
    if (c >= nc || b >= nb || a >= na) return;
    const long long fs = g.fstride;
    long long fi;
    double *const *mS;
    double *const *pS;
    long long plus, dn, dt1, dt2;
    double rdn, rt1, rt2;
    if (N == 1) {
        fi = ((long long)a * nb + b) * nc + c;
        mS = f.x[0]; pS = f.x[1];
        plus = g.idx(a + 1, b + 1, c + 1); dn = g.pi; dt1 = g.pk; dt2 = 1;
        rdn = kc.rdx; rt1 = kc.r4dy; rt2 = kc.r4dz;
    } else if (N == 2) {
        fi = ((long long)a * nb + b) * nc + c;
        mS = f.y[0]; pS = f.y[1];
        plus = g.idx(a + 1, b + 1, c + 1); dn = g.pk; dt1 = g.pi; dt2 = 1;
        rdn = kc.rdy; rt1 = kc.r4dx; rt2 = kc.r4dz;
    } else {
        fi = ((long long)a * nb + b) * nc + c;
        mS = f.z[0]; pS = f.z[1];
        plus = g.idx(a + 1, b + 1, c + 1); dn = 1; dt1 = g.pi; dt2 = g.pk;
        rdn = kc.rdz; rt1 = kc.r4dx; rt2 = kc.r4dy;
    }
    const long long minus = plus - dn;
    // the neighbours read: plus and minus, each with both tangential offsets
    if (!FSL_SPAN(plus, -dn - (dt1 > dt2 ? dt1 : dt2), dt1 > dt2 ? dt1 : dt2, fs)) return;
    fi = FSL_FACE(fi, (long long)na * nb * nc);
    double Lm[5], Rp[5];
#pragma unroll
    for (int q = 0; q < 5; q++) { Lm[q] = mS[q][fi]; Rp[q] = pS[q][fi]; }
    double Rho, P, vel[3];
    riemann<double, N>(Lm, Rp, Rho, P, vel);
    double vp[3], vm[3], Tp, Tm;
    vel_div(u[plus], u[fs + plus], u[2 * fs + plus], u[3 * fs + plus], u[4 * fs + plus], vp, Tp);
    vel_div(u[minus], u[fs + minus], u[2 * fs + minus], u[3 * fs + minus], u[4 * fs + minus], vm, Tm);
    // tangential neighbours: P/M = plus/minus cell, h/l = +/- tangential offset
    double Ph1[3], Mh1[3], Pl1[3], Ml1[3], Ph2[3], Mh2[3], Pl2[3], Ml2[3];
#define LOADV(dst, at) vel_rcp(u[at], u[fs + (at)], u[2 * fs + (at)], u[3 * fs + (at)], dst)
    LOADV(Ph1, plus + dt1); LOADV(Mh1, minus + dt1); LOADV(Pl1, plus - dt1); LOADV(Ml1, minus - dt1);
    LOADV(Ph2, plus + dt2); LOADV(Mh2, minus + dt2); LOADV(Pl2, plus - dt2); LOADV(Ml2, minus - dt2);
#undef LOADV
    // g[a][b] = d u_a / d x_b
    double gr[3][3];
    const int n0 = N - 1;
    const int t1 = (N == 1) ? 1 : 0;   // first tangential axis
    const int t2 = (N == 3) ? 1 : 2;   // second tangential axis
#pragma unroll
    for (int q = 0; q < 3; q++) {
        gr[q][n0] = (vp[q] - vm[q]) * rdn;
        gr[q][t1] = (Ph1[q] + Mh1[q] - Pl1[q] - Ml1[q]) * rt1;
        gr[q][t2] = (Ph2[q] + Mh2[q] - Pl2[q] - Ml2[q]) * rt2;
    }
    // SGS viscosity at the face: x uses the two adjacent cells (:191); the y
    // and z sweeps average the plus cell with its x-neighbour (:360, :531).
    double mu_T;
    if (sgs == FSL_SGS_STATIC) mu_T = static_mu_t<double>(gr, 0.5 * (u[plus] + u[minus]), kc.CsDD);
    else if (sgs == FSL_SGS_NONE) mu_T = 0.0;
    else mu_T = 0.5 * (mu[plus] + mu[plus - g.pi]);
    double F[5];
    face_flux<double, N>(Rho, P, vel, gr, vp, vm, Tp, Tm, kc.mu_L, mu_T, kc.lambda_L, kc.cp_Pr_T, rdn, F);
#pragma unroll
    for (int q = 0; q < 5; q++) mS[q][fi] = F[q];
}

// ---------------------------------------------------------------------------
// A7 TVD Runge-Kutta (src/evolution.c:15-245).  mode: 1..3 = RK3 stage,
// 4 = the nStages == 2 chain of stage 1, 5 = the chain of stage 2 (RK2 stage
// 2 followed by RK3 stage 2 on the updated U, src/evolution.c:19-23).
// ---------------------------------------------------------------------------
__global__ void k_evolution(Grid g, int mode, const DevScalars *__restrict__ ds, double *__restrict__ U,
                            double *__restrict__ Up, Faces f)
{
    const int L = g.L, H = g.H, D = g.D;
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > D || j > H) return;
    const double dtx = ds->dtx, dty = ds->dty, dtz = ds->dtz;
    const double one_third = 1. / 3., two_thirds = 2. / 3.;
    const long long fs = g.fstride, c = FSL_CELL(g.idx(i, j, k), fs);
    const long long xm = ixf(L, H, D, i - 1, j - 1, k - 1), xp = ixf(L, H, D, i, j - 1, k - 1);
    const long long ym = iyf(L, H, D, i - 1, j - 1, k - 1), yp = iyf(L, H, D, i - 1, j, k - 1);
    const long long zm = izf(L, H, D, i - 1, j - 1, k - 1), zp = izf(L, H, D, i - 1, j - 1, k);
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const double X = dtx * (f.x[0][q][xm] - f.x[0][q][xp]);
        const double Y = dty * (f.y[0][q][ym] - f.y[0][q][yp]);
        const double Z = dtz * (f.z[0][q][zm] - f.z[0][q][zp]);
        double *u = U + q * fs, *up = Up + q * fs;
        if (mode == 1 || mode == 4) {
            up[c] = u[c] + X + Y + Z;
        } else if (mode == 2) {
            up[c] = 0.75 * u[c] + 0.25 * (up[c] + X + Y + Z);
        } else if (mode == 3) {
            u[c] = one_third * u[c] + two_thirds * (up[c] + X + Y + Z);
        } else { // mode 5
            const double un = 0.5 * (u[c] + up[c] + X + Y + Z);
            u[c] = un;
            up[c] = 0.75 * un + 0.25 * (up[c] + X + Y + Z);
        }
    }
}

// ---------------------------------------------------------------------------
// A8 Courant maximum (src/helpers.c:23-52).  NaN never wins a comparison, as
// in the reference's `(CoNum = U*deltaT_X) > maxCo`, so the maximum is
// independent of reduction order.
// ---------------------------------------------------------------------------
__global__ void k_courant_partial(Grid g, Consts kc, const double *__restrict__ U,
                                  const DevScalars *__restrict__ ds, double *__restrict__ partials,
                                  DevScalars *__restrict__ dsw, int i0, int i1)
{
    const int H = g.H, D = g.D;
    const long long n = (long long)(i1 - i0 + 1) * H * D; // planes i0..i1
    const long long fs = g.fstride;
    const double dtx = ds->dtx, dty = ds->dty, dtz = ds->dtz;
    double m = 0.0;
    unsigned bad = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % D) + 1;
        const long long r = t / D;
        const int j = (int)(r % H) + 1;
        const int i = (int)(r / H) + i0;
        const long long c = FSL_CELL(g.idx(i, j, k), g.fstride);
        const double R = U[c];
        const double Co = cell_courant(kc.cfl_mode, R, U[fs + c], kc.cfl_mode == FSL_CFL_ACOUSTIC ? U[2 * fs + c] : 0.,
                                       kc.cfl_mode == FSL_CFL_ACOUSTIC ? U[3 * fs + c] : 0.,
                                       kc.cfl_mode == FSL_CFL_ACOUSTIC ? U[4 * fs + c] : 0., dtx, dty, dtz);
        m = (Co > m) ? Co : m;
        if (!(R > 0.0)) bad = 1;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, m, o);
        m = (x > m) ? x : m;
    }
    __shared__ double sm[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sm[w] = m;
    if (bad) atomicOr(&dsw->status, 2u);
    __syncthreads();
    if (w == 0) {
        m = (l < (int)(blockDim.x >> 5)) ? sm[l] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_xor_sync(0xffffffffu, m, o);
            m = (x > m) ? x : m;
        }
        if (l == 0) partials[blockIdx.x] = m;
    }
}

// dt rescale of src/helpers.c:47-50; clears the fused accumulator for the
// next stage 3
__device__ __forceinline__ void apply_courant(const Consts &kc, double maxCo, DevScalars *ds)
{
    double dt = ds->dt;
    dt *= (kc.maxCoNum / maxCo);
    ds->dt = dt;
    ds->dtx = dt / kc.deltaX;
    ds->dty = dt / kc.deltaY;
    ds->dtz = dt / kc.deltaZ;
    ds->maxCo = maxCo;
    ds->co_bits = 0ull;
    if (!(maxCo > 0.0) || !isfinite(maxCo) || !isfinite(dt)) ds->status |= 1u;
}

// Final reduction and the dt rescale of src/helpers.c:47-50.
__global__ void k_courant_final(Consts kc, const double *__restrict__ partials, int np, DevScalars *ds)
{
    double m = 0.0;
    for (int t = threadIdx.x; t < np; t += blockDim.x) {
        const double x = partials[t];
        m = (x > m) ? x : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double x = __shfl_xor_sync(0xffffffffu, m, o);
        m = (x > m) ? x : m;
    }
    __shared__ double sm[32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sm[w] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        m = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) m = (sm[q] > m) ? sm[q] : m;
        apply_courant(kc, m, ds);
    }
}

// The maximum of the partials as the accumulator's bit pattern, without the
// dt update (the Courant maximum of a slab, to be combined across slabs).
__global__ void k_courant_to_bits(const double *__restrict__ partials, int np, DevScalars *ds)
{
    if (threadIdx.x != 0) return;
    double m = 0.0;
    for (int t = 0; t < np; t++) m = (partials[t] > m) ? partials[t] : m;
    ds->co_bits = (unsigned long long)__double_as_longlong(m);
}

// The same dt update from the maximum the fused stage 3 of the previous step
// accumulated over the state it wrote (that state is this step's U^n).
__global__ void k_courant_apply(Consts kc, DevScalars *ds)
{
    if (threadIdx.x == 0) apply_courant(kc, __longlong_as_double((long long)ds->co_bits), ds);
}

// Per y row: sums over the x-z plane of a, b, (a-b)^2 and b^2 (two padded
// fields) -- the judgement of the learned closure, over the band two cells
// away from every boundary (nearer, the dynamic procedure's values carry the
// zero padding of the reference's test filter); rows outside it are zero.
template <typename TA, typename TB>
__global__ void k_judge_rows(Grid g, const TA *__restrict__ a, const TB *__restrict__ b,
                             double *__restrict__ rows)
{
    const int j = blockIdx.x + 1;
    const int bL = g.L - 4, bD = g.D - 4;
    const long long n = (j >= 3 && j <= g.H - 2) ? (long long)bL * bD : 0;
    double s[4] = {0, 0, 0, 0};
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = (int)(t % bD) + 3;
        const int i = (int)(t / bD) + 3;
        const long long c = FSL_CELL(g.idx(i, j, k), g.fstride);
        const double x = a[c], y = b[c];
        s[0] += x; s[1] += y; s[2] += (x - y) * (x - y); s[3] += y * y;
    }
    __shared__ double sm[4][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 4; q++) {
        double x = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (l == 0) sm[q][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double x = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sm[threadIdx.x][q];
        rows[(long long)blockIdx.x * 4 + threadIdx.x] = x;
    }
}

// ---------------------------------------------------------------------------
// state transfer and diagnostics
// ---------------------------------------------------------------------------
__global__ void k_state_scatter(Grid g, double *__restrict__ dst, const double *__restrict__ packed, int i0, int ni)
{
    const long long n = (long long)ni * g.H * 5 * g.D;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.D);
        long long r = t / g.D;
        const int v = (int)(r % 5); r /= 5;
        const int j = (int)(r % g.H);
        const int i = (int)(r / g.H);
        dst[v * g.fstride + FSL_CELL(g.idx(i + i0, j + 1, k + 1), g.fstride)] = packed[t];
    }
}

// planes i0 .. i0+ni-1 (1-based interior planes) in the state layout
__global__ void k_state_gather(Grid g, const double *__restrict__ src, double *__restrict__ packed, int i0, int ni)
{
    const long long n = (long long)ni * g.H * 5 * g.D;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.D);
        long long r = t / g.D;
        const int v = (int)(r % 5); r /= 5;
        const int j = (int)(r % g.H);
        const int i = (int)(r / g.H);
        packed[t] = src[v * g.fstride + FSL_CELL(g.idx(i + i0, j + 1, k + 1), g.fstride)];
    }
}

// Deterministic block partial sums of the five conserved variables over
// the interior planes i0 .. i0+ni-1.
__global__ void k_sums_partial(Grid g, int i0, int ni, const double *__restrict__ U, double *__restrict__ partials)
{
    const long long n = (long long)ni * g.H * g.D;
    double s[5] = {0, 0, 0, 0, 0};
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(t % g.D) + 1;
        const long long r = t / g.D;
        const int j = (int)(r % g.H) + 1;
        const int i = (int)(r / g.H) + i0;
        const long long c = FSL_CELL(g.idx(i, j, k), g.fstride);
#pragma unroll
        for (int q = 0; q < 5; q++) s[q] += U[q * g.fstride + c];
    }
    __shared__ double sm[5][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        double x = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (l == 0) sm[q][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double x = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sm[threadIdx.x][q];
        partials[blockIdx.x * 5 + threadIdx.x] = x;
    }
}

__global__ void k_sums_final(const double *__restrict__ partials, int np, double vol, double *__restrict__ out)
{
    if (threadIdx.x < 5) {
        double x = 0;
        for (int b = 0; b < np; b++) x += partials[b * 5 + threadIdx.x];
        out[threadIdx.x] = x * vol;
    }
}

// One block per y row: sums over the x-z plane (interior planes i0 ..
// i0+ni-1) of rho, rho u, rho v, rho w, rho uu, rho vv, rho ww, rho uv.
__global__ void k_plane_sums(Grid g, int i0, int ni, const double *__restrict__ U, double *__restrict__ rows)
{
    const int j = blockIdx.x + 1;
    const long long n = (long long)ni * g.D;
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long t = threadIdx.x; t < n; t += blockDim.x) {
        const int k = (int)(t % g.D) + 1;
        const int i = (int)(t / g.D) + i0;
        const long long c = FSL_CELL(g.idx(i, j, k), g.fstride);
        const double r = U[c], u = U[g.fstride + c] / r, v = U[2 * g.fstride + c] / r,
                     w = U[3 * g.fstride + c] / r;
        s[0] += r; s[1] += r * u; s[2] += r * v; s[3] += r * w;
        s[4] += r * u * u; s[5] += r * v * v; s[6] += r * w * w; s[7] += r * u * v;
    }
    __shared__ double sm[8][32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int q = 0; q < 8; q++) {
        double x = s[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (l == 0) sm[q][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 8) {
        double x = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); q++) x += sm[threadIdx.x][q];
        rows[(long long)blockIdx.x * 8 + threadIdx.x] = x;
    }
}

inline dim3 cells_grid(const Grid &g, dim3 b, int ni, int nj, int nk)
{
    return dim3((nk + b.x - 1) / b.x, (nj + b.y - 1) / b.y, ni);
}

} // namespace

// ---- launchers -------------------------------------------------------------

void launch_ghost(Ctx &c, double *cur)
{
    const Grid &g = c.g;
    const long long n = 2LL * (g.H + 2) * (g.D + 2) + 2LL * g.L * (g.D + 2) + 2LL * g.L * g.H;
    prof_begin(c, FSL_K_BC);
    k_ghost<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(g, c.k.setup, cur);
    prof_end(c, FSL_K_BC, 1);
}

void launch_recon(Ctx &c, const double *cur)
{
    const Grid &g = c.g;
    dim3 b(32, 4, 1);
    prof_begin(c, FSL_K_RECON);
    if (c.p.recon == FSL_RECON_PPM) k_recon<true><<<cells_grid(g, b, g.L, g.H, g.D), b, 0, c.stream>>>(g, cur, c.f);
    else k_recon<false><<<cells_grid(g, b, g.L, g.H, g.D), b, 0, c.stream>>>(g, cur, c.f);
    prof_end(c, FSL_K_RECON, 1);
}

void launch_ifbc(Ctx &c, const Disturb &d)
{
    const Grid &g = c.g;
    const long long n = (long long)g.H * g.D + (long long)g.L * g.D + (long long)g.L * g.H;
    prof_begin(c, FSL_K_BC);
    k_ifbc<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(g, c.k.setup, c.k.BL_HIG, d, c.f);
    prof_end(c, FSL_K_BC, 1);
}

void launch_fluxes(Ctx &c, const double *cur)
{
    const Grid &g = c.g;
    dim3 b(32, 4, 1);
    prof_begin(c, FSL_K_FLUX);
    k_flux<1><<<cells_grid(g, b, g.L + 1, g.H, g.D), b, 0, c.stream>>>(g, c.k, cur, c.mu, c.f, c.p.sgs);
    k_flux<2><<<cells_grid(g, b, g.L, g.H + 1, g.D), b, 0, c.stream>>>(g, c.k, cur, c.mu, c.f, c.p.sgs);
    k_flux<3><<<cells_grid(g, b, g.L, g.H, g.D + 1), b, 0, c.stream>>>(g, c.k, cur, c.mu, c.f, c.p.sgs);
    prof_end(c, FSL_K_FLUX, 3);
}

void launch_evolution(Ctx &c, int nstages, int stage)
{
    const Grid &g = c.g;
    int mode = stage >= 3 ? 3 : stage;
    if (nstages == 2) mode = (stage == 1) ? 4 : 5;
    dim3 b(32, 4, 1);
    prof_begin(c, FSL_K_EVOL);
    k_evolution<<<cells_grid(g, b, g.L, g.H, g.D), b, 0, c.stream>>>(g, mode, c.ds, c.U, c.Up, c.f);
    prof_end(c, FSL_K_EVOL, 1);
}

void launch_dynsmag(Ctx &c, const double *U, float *cd)
{
    const DynScratch &s = c.dyn;
    const dyn::Scratch3<double> sc{s.vel, s.F, s.A, s.S};
    prof_begin(c, FSL_K_SGS);
    dyn::sequence_fused<double>(c.g, c.k, sc, U, c.mu, cd, c.stream);
    prof_end(c, FSL_K_SGS, 4);
}

void launch_courant(Ctx &c)
{
    const Grid &g = c.g;
    prof_begin(c, FSL_K_CFL);
    k_courant_partial<<<c.npartials, 256, 0, c.stream>>>(g, c.k, c.U, c.ds, c.partials, c.ds, c.co_i0, c.co_i1);
    k_courant_final<<<1, 1024, 0, c.stream>>>(c.k, c.partials, c.npartials, c.ds);
    prof_end(c, FSL_K_CFL, 2);
}

void launch_courant_to_bits(Ctx &c)
{
    prof_begin(c, FSL_K_CFL);
    k_courant_partial<<<c.npartials, 256, 0, c.stream>>>(c.g, c.k, c.U, c.ds, c.partials, c.ds, c.co_i0, c.co_i1);
    k_courant_to_bits<<<1, 32, 0, c.stream>>>(c.partials, c.npartials, c.ds);
    prof_end(c, FSL_K_CFL, 2);
}

void launch_courant_apply(Ctx &c)
{
    prof_begin(c, FSL_K_CFL);
    k_courant_apply<<<1, 32, 0, c.stream>>>(c.k, c.ds);
    prof_end(c, FSL_K_CFL, 1);
}

void launch_state_scatter(Ctx &c, double *dst, const double *packed, int i0, int ni)
{
    if (ni <= 0) return;
    prof_begin(c, FSL_K_OTHER);
    k_state_scatter<<<148 * 8, 256, 0, c.stream>>>(c.g, dst, packed, i0, ni);
    prof_end(c, FSL_K_OTHER, 1);
}

void launch_state_gather(Ctx &c, const double *src, double *packed, int i0, int ni)
{
    if (ni <= 0) return;
    prof_begin(c, FSL_K_OTHER);
    k_state_gather<<<148 * 8, 256, 0, c.stream>>>(c.g, src, packed, i0, ni);
    prof_end(c, FSL_K_OTHER, 1);
}

void launch_sums(Ctx &c, const double *U, int i0, int ni, double *out5)
{
    const int nb = 148 * 4;
    prof_begin(c, FSL_K_OTHER);
    k_sums_partial<<<nb, 256, 0, c.stream>>>(c.g, i0, ni, U, c.partials);
    const double vol = c.p.deltaX * c.p.deltaY * c.p.deltaZ;
    k_sums_final<<<1, 32, 0, c.stream>>>(c.partials, nb, vol, out5);
    prof_end(c, FSL_K_OTHER, 2);
}

template <typename TA, typename TB> static void judge_rows_t(Ctx &c, const TA *a, const TB *b, double *rows)
{
    prof_begin(c, FSL_K_OTHER);
    k_judge_rows<TA, TB><<<c.g.H, 256, 0, c.stream>>>(c.g, a, b, rows);
    prof_end(c, FSL_K_OTHER, 1);
}
void launch_judge_rows(Ctx &c, const float *a, const float *b, double *rows) { judge_rows_t(c, a, b, rows); }
void launch_judge_rows(Ctx &c, const float *a, const double *b, double *rows) { judge_rows_t(c, a, b, rows); }
void launch_judge_rows(Ctx &c, const double *a, const double *b, double *rows) { judge_rows_t(c, a, b, rows); }

void launch_plane_sums(Ctx &c, const double *U, int i0, int ni, double *rows)
{
    prof_begin(c, FSL_K_OTHER);
    k_plane_sums<<<c.g.H, 256, 0, c.stream>>>(c.g, i0, ni, U, rows);
    prof_end(c, FSL_K_OTHER, 1);
}

} // namespace fsl

// ---------------------------------------------------------------------------
// Allocation-free SGS viscosity (fsl_dynamic_smagorinsky_noalloc).
//
// Callers that cannot allocate device memory hand in their own input and
// output buffers; the procedure's 40 scratch fields live in this fixed static
// device array instead of cudaMalloc'd memory.  Every GPU that loads the
// library holds the array until the process exits.  On the host the symbol
// name only stands in for the array; the device address is looked up once per
// device with cudaGetSymbolAddress (that device current) and cached.
// ---------------------------------------------------------------------------
#include <cmath>
#include <mutex>

static __device__ __align__(256) double fsl_noalloc_scratch[FSL_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double *g_noalloc_ptr[kNoallocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.
int noalloc_scratch(double **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FSL_ERR_NODEVICE;
    if (dev < 0 || dev >= kNoallocMaxDevices) return FSL_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, fsl_noalloc_scratch);
        if (e != cudaSuccess || !p) return FSL_ERR_CUDA;
        g_noalloc_ptr[dev] = static_cast<double *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return FSL_OK;
}

// The dynamic procedure's unfused nine-launch sequence (dyn::sequence: the
// seven-pass filters and the coefficient, each field in its own scratch
// array), on explicit buffers and stream.  The context path runs the fused
// form (dyn::sequence_fused) on less scratch; both give the same bits.
void noalloc_dyn_sequence(const fsl::Grid &g, const fsl::Consts &k, const fsl::dyn::Scratch<double> &s,
                          const double *U, double *mu, cudaStream_t st)
{
    fsl::dyn::sequence<double>(g, k, s, U, mu, nullptr, st);
}

} // namespace

extern "C" int fsl_dynamic_smagorinsky_noalloc(const double *U, double *mu, int LEN, int HIG, int DEP,
                                                double deltaX, double deltaY, double deltaZ, void *stream)
{
    if (!U || !mu || LEN < 2 || HIG < 2 || DEP < 2 || !(deltaX > 0) || !(deltaY > 0) || !(deltaZ > 0))
        return FSL_ERR_ARG;
    // each extent widened before the +2, so no int arithmetic can overflow
    const long long n = ((long long)LEN + 2) * ((long long)HIG + 2) * ((long long)DEP + 2);
    if (n <= 0) return FSL_ERR_ARG;
    if (n > (long long)FSL_NOALLOC_MAX_CELLS) return FSL_ERR_TOO_LARGE;
    // an error left pending by the caller's earlier work is not this call's:
    // report it without clearing it and without starting any work
    if (cudaPeekAtLastError() != cudaSuccess) return FSL_ERR_CUDA;
    double *s = nullptr;
    int rc = noalloc_scratch(&s);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the scratch address belongs to the current device: a stream of another
    // device would run the work against that device's copy of the array
    if (st) {
        int sdev = -1, dev = -1;
        if (cudaStreamGetDevice(st, &sdev) != cudaSuccess || cudaGetDevice(&dev) != cudaSuccess) return FSL_ERR_ARG;
        if (sdev != dev) return FSL_ERR_ARG;
    }
    fsl::Grid g;
    g.L = LEN; g.H = HIG; g.D = DEP;
    g.pk = DEP + 2;
    g.pi = (long long)(DEP + 2) * (HIG + 2);
    g.off = 0;
    g.fstride = n;
    // derived constants exactly as fsl_init computes them (src/initialize.c:67-94)
    fsl::Consts k{};
    k.r4dx = 1. / (4 * deltaX); k.r4dy = 1. / (4 * deltaY); k.r4dz = 1. / (4 * deltaZ);
    k.r2dx = k.r4dx + k.r4dx; k.r2dy = k.r4dy + k.r4dy; k.r2dz = k.r4dz + k.r4dz;
    k.DD = pow(deltaX * deltaY * deltaZ, 0.666666666666667);
    fsl::dyn::Scratch<double> d;
    d.vel = s; d.t1 = s + 3 * n; d.t2 = s + 12 * n; d.A = s + 21 * n;
    d.Lst = s + 27 * n; d.B = s + 33 * n; d.S = s + 39 * n;
    // zero bands of the filter passes and the A ghost layer must start at 0;
    // the previous call left its values in the shared scratch
    if (cudaMemsetAsync(s, 0, (size_t)(40 * n) * sizeof(double), st) != cudaSuccess) return FSL_ERR_CUDA;
    if (cudaMemsetAsync(mu, 0, (size_t)n * sizeof(double), st) != cudaSuccess) return FSL_ERR_CUDA;
    noalloc_dyn_sequence(g, k, d, U, mu, st);
    if (cudaGetLastError() != cudaSuccess) return FSL_ERR_CUDA;
    return FSL_OK;
}
