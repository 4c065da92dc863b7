// fsl_stage.cuh -- fused RK3 stage kernel and boundary-face pass, templated on
// the compute type T.  Instantiated for T = double (fsl_fused.cu, compiled
// with --fmad=false: the plain method, bit-identical to the reference) and
// T = float (fsl_fused32.cu: FP32 bulk, FP64 stage accumulation).
//
// Decomposition ("2.5-D" streaming): a block owns a tile of (TJE-2) x 30
// cell columns in (y, z) plus a one-cell halo ring (TJE rows = warps, 32
// lanes along the contiguous k axis) and marches along x over `seg` planes.
// Per plane it stages in shared memory the current-stage state (two planes,
// halo 2), the two velocity forms the viscous stencil reads (src/fluxes.c
// divides for the two cells adjacent to a face, :117-122, and multiplies by a
// reciprocal for the eight tangential neighbours, :124-142), temperature and
// the face-averaged SGS viscosity.  Every face flux of the tile is computed
// once (x faces in registers carried along the march, y faces through shared
// memory, z faces through warp shuffles); the state is read once and the
// stage result written once.  Plane i+2 is fetched into registers at the top
// of iteration i and stored to shared memory at its end, hiding the load
// latency behind the flux work.  Domain-boundary faces take their outer state
// from the boundary pass (k_bface), which applies the reference's interface
// rules (src/bounCondOnInterfaces.c:11-110) to the reconstructed boundary cells.
#pragma once

#include "fsl_check.cuh"
#include "fsl_internal.h"
#include "fsl_phys.cuh"

namespace fsl {
namespace stage {

template <typename T> struct BF {
    T *x0, *xL, *y0, *yH, *z0, *zD;
};

template <typename T>
__device__ __forceinline__ void load5(const double *__restrict__ u, long long fs, long long c, T *v)
{
#pragma unroll
    for (int q = 0; q < 5; q++) v[q] = T(u[q * fs + FSL_CELL(c, fs)]);
}

// reconstruction sweep DIR (0 x, 1 y, 2 z) of the padded cell c
template <typename T, int DIR>
__device__ __forceinline__ void recon_at(const Grid &g, const double *__restrict__ u, long long c, T *hi, T *lo)
{
    const long long fs = g.fstride;
    CellC<T> cc;
    load5(u, fs, c, cc.u);
    cell_consts(cc);
    const long long d = DIR == 0 ? g.pi : DIR == 1 ? (long long)g.pk : 1LL;
    const int p1 = DIR == 0 ? 1 : DIR == 1 ? 2 : 3;
    const int p2 = DIR == 0 ? 2 : DIR == 1 ? 3 : 1;
    const int p3 = DIR == 0 ? 3 : DIR == 1 ? 1 : 2;
    T fw[5], bw[5];
    const long long cf = FSL_CELL(c + d, fs), cb = FSL_CELL(c - d, fs);
    fw[0] = T(u[cf]); fw[1] = T(u[p1 * fs + cf]); fw[2] = T(u[p2 * fs + cf]);
    fw[3] = T(u[p3 * fs + cf]); fw[4] = T(u[4 * fs + cf]);
    bw[0] = T(u[cb]); bw[1] = T(u[p1 * fs + cb]); bw[2] = T(u[p2 * fs + cb]);
    bw[3] = T(u[p3 * fs + cb]); bw[4] = T(u[4 * fs + cb]);
    if (DIR == 0) recon_x(cc, fw, bw, hi, lo);
    else if (DIR == 1) recon_y(cc, fw, bw, hi, lo);
    else recon_z(cc, fw, bw, hi, lo);
}

// PPM x-sweep of the padded cell c (planes c-2 .. c+2 from global memory)
template <typename T>
__device__ __forceinline__ void ppm_at_x(const Grid &g, const double *__restrict__ u, long long c, T *hi, T *lo)
{
    const long long fs = g.fstride, d = g.pi;
    CellC<T> cc;
    T m2[5], m1[5], p1[5], p2[5];
    load5(u, fs, c, cc.u);
    load5(u, fs, c - 2 * d, m2);
    load5(u, fs, c - d, m1);
    load5(u, fs, c + d, p1);
    load5(u, fs, c + 2 * d, p2);
    cell_consts(cc);
    ppm_x(cc, m2, m1, p1, p2, hi, lo);
}

// Outer states of one domain-boundary face (src/bounCondOnInterfaces.c:11-110):
// face t of the x (HIG DEP), y (LEN DEP) and z (LEN HIG) boundary lists.
// Not inlined: the boundary pass and the persistent multi-domain stage
// kernel run this one compiled body, so their FP32 results agree bit for bit.
template <typename T>
__device__ __noinline__ void bface_one(Grid g, int setup, int BL_HIG, Disturb d, const double *__restrict__ u,
                                       BF<T> bf, long long t)
{
    const int L = g.L, H = g.H, D = g.D;
    const long long nx = (long long)H * D, ny = (long long)L * D, nz = (long long)L * H;
    const bool spatial = (setup == FSL_SETUP_SPATIAL);
    typedef Kc<T> kc;
    T hi[5], lo[5];
    if (t < nx) {
        const int jf = (int)(t / D), kf = (int)(t % D);
        const int j = jf + 1, k = kf + 1;
        const long long fo = t;
        if (spatial) {
            // inflow profile in the reference's FP64 arithmetic (:17-60)
            const double P = 100000., R = 1.0;
            double U, V = 0., W = 0., v[5];
            if (jf < H / 2) {
                U = 76.4;
                v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.; v[4] = P / 0.4 + 0.5 * R * (U * U);
            } else if (jf < H / 2 + BL_HIG) {
                const unsigned ku = (unsigned)kf;
                bool dist;
                if (d.k_max > d.k_min) dist = (ku >= d.k_min && ku < d.k_max);
                else dist = !(ku >= d.k_max && ku < d.k_min);
                if (dist) { U = 200. + d.Ud; V = d.Vd; W = d.Wd; }
                else { U = 200.; V = W = 0.; }
                v[0] = R; v[1] = R * U; v[2] = R * V; v[3] = R * W;
                v[4] = P / 0.4 + 0.5 * R * (U * U + V * V + W * W);
            } else {
                U = 200.;
                v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.; v[4] = P / 0.4 + 0.5 * R * (U * U);
            }
#pragma unroll
            for (int q = 0; q < 5; q++) bf.x0[q * nx + FSL_FACE(fo, nx)] = T(v[q]);
            // :62-71 outflow from the minus state of face LEN
            recon_at<T, 0>(g, u, g.idx(L, j, k), hi, lo);
            const T r = hi[0], mu_ = hi[1], mv = hi[2], mw = hi[3];
            const T P_ = T(100000.);
            const long long fc = FSL_FACE(fo, nx);
            bf.xL[fc] = r; bf.xL[nx + fc] = mu_; bf.xL[2 * nx + fc] = mv; bf.xL[3 * nx + fc] = mw;
            bf.xL[4 * nx + fc] = P_ / kc::K_1 + T(0.5) * (mu_ * mu_ + mv * mv + mw * mw) / r;
        } else { // periodic x, the reference's z rule (:94-109)
            recon_at<T, 0>(g, u, g.idx(L, j, k), hi, lo);
#pragma unroll
            for (int q = 0; q < 5; q++) bf.x0[q * nx + FSL_FACE(fo, nx)] = hi[q];
            recon_at<T, 0>(g, u, g.idx(1, j, k), hi, lo);
#pragma unroll
            for (int q = 0; q < 5; q++) bf.xL[q * nx + FSL_FACE(fo, nx)] = lo[q];
        }
    } else if ((t -= nx) < ny) { // :75-90
        const int i = (int)(t / D) + 1, k = (int)(t % D) + 1;
        recon_at<T, 1>(g, u, g.idx(i, 1, k), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.y0[q * ny + FSL_FACE(t, ny)] = (q == 2 && spatial) ? -lo[q] : lo[q];
        recon_at<T, 1>(g, u, g.idx(i, H, k), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.yH[q * ny + FSL_FACE(t, ny)] = (q == 2 && spatial) ? -hi[q] : hi[q];
    } else if ((t -= ny) < nz) { // :94-109
        const int i = (int)(t / H) + 1, j = (int)(t % H) + 1;
        recon_at<T, 2>(g, u, g.idx(i, j, D), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.z0[q * nz + FSL_FACE(t, nz)] = hi[q];
        recon_at<T, 2>(g, u, g.idx(i, j, 1), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.zD[q * nz + FSL_FACE(t, nz)] = lo[q];
    }
}

template <typename T>
__global__ void k_bface(Grid g, int setup, int BL_HIG, Disturb d, const double *__restrict__ u, BF<T> bf)
{
    const long long n = (long long)g.H * g.D + (long long)g.L * g.D + (long long)g.L * g.H;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) bface_one<T>(g, setup, BL_HIG, d, u, bf, t);
}

template <typename T, int TJE, bool PPM = false> struct Smem {
    static constexpr int HW = PPM ? 2 : 1; // y/z halo width of the state planes
    static constexpr int NS = PPM ? 4 : 2; // x-planes in the state ring
    // current-stage state: planes i, i+1 (PPM: i-1 .. i+2) as a ring, with
    // HW halo rows and lanes
    T U[NS][TJE + 2 * HW][32 + 2 * HW][5];
    T R[3][TJE][32][3];     // velocities by reciprocal, planes i-1, i, i+1 (ring)
    T Dv[2][TJE][32][5];    // velocities by division, temperature, mu face average, planes i, i+1
    T Lo[TJE][32][5];       // y sweep: state on the face below each cell
    T Fy[TJE][32][5];       // y flux on the face above each row
};

template <typename T> struct Args {
    const double *cur; // current-stage state, ghost layer filled
    const double *un;  // U^n
    double *out;
    const T *mu;
    BF<T> bf;
    const DevScalars *ds;
    unsigned long long *co; // non-null: accumulate the Courant maximum of `out` (stage 3)
    int co_i0, co_i1;       // over planes co_i0..co_i1 only
    unsigned int *status;   // bit 1 set on a non-positive output density (with co)
    int stage;
    int seg;
    // non-null (full-lane tile, temporal setup): also write the FP32 velocities
    // of `out`, ghost cells included, as the closure's velocity pass forms them
    float *vel;
};

// Own column of plane `pl` (and, on the tile edge, the halo neighbour the y
// and z sweeps need) from global memory into registers.
// Kept in the storage type (FP64) while in flight: a conversion at load
// time would wait on the load immediately.
struct PlaneLoad {
    double own[5], halo[5], halo2[5]; // halo2: the second halo cell (PPM)
};

template <typename T, int TJE, bool PPM>
__device__ __forceinline__ void plane_issue(const Grid &g, const double *__restrict__ cu, int pl, int r, int l, int j,
                                            int k, bool live, PlaneLoad &p)
{
    const long long fs = g.fstride;
    if (!live || pl > g.L + 1) return;
    const long long c = g.idx(pl, j, k);
    load5(cu, fs, c, p.own);
    if (r == 0 && j >= 1) {
        load5(cu, fs, c - g.pk, p.halo);
        if (PPM && j >= 2) load5(cu, fs, c - 2 * g.pk, p.halo2);
    } else if (r == TJE - 1 && j <= g.H) {
        load5(cu, fs, c + g.pk, p.halo);
        if (PPM && j <= g.H - 1) load5(cu, fs, c + 2 * g.pk, p.halo2);
    } else if (l == 0 && k >= 1) {
        load5(cu, fs, c - 1, p.halo);
        if (PPM && k >= 2) load5(cu, fs, c - 2, p.halo2);
    } else if (l == 31 && k <= g.D) {
        load5(cu, fs, c + 1, p.halo);
        if (PPM && k <= g.D - 1) load5(cu, fs, c + 2, p.halo2);
    }
}

template <typename T, int TJE, bool PPM>
__device__ __forceinline__ void plane_store(Smem<T, TJE, PPM> &s, int slot, int r, int l, int j, int k, int H, int D,
                                            bool live, const PlaneLoad &p)
{
    constexpr int HW = Smem<T, TJE, PPM>::HW;
    if (!live) return;
#pragma unroll
    for (int q = 0; q < 5; q++) s.U[slot][r + HW][l + HW][q] = T(p.own[q]);
    T *h = nullptr, *h2 = nullptr;
    if (r == 0 && j >= 1) {
        h = s.U[slot][HW - 1][l + HW];
        if (PPM && j >= 2) h2 = s.U[slot][0][l + HW];
    } else if (r == TJE - 1 && j <= H) {
        h = s.U[slot][TJE + HW][l + HW];
        if (PPM && j <= H - 1) h2 = s.U[slot][TJE + HW + 1][l + HW];
    } else if (l == 0 && k >= 1) {
        h = s.U[slot][r + HW][HW - 1];
        if (PPM && k >= 2) h2 = s.U[slot][r + HW][0];
    } else if (l == 31 && k <= D) {
        h = s.U[slot][r + HW][32 + HW];
        if (PPM && k <= D - 1) h2 = s.U[slot][r + HW][33 + HW];
    }
    if (h) {
#pragma unroll
        for (int q = 0; q < 5; q++) h[q] = T(p.halo[q]);
    }
    if (PPM && h2) {
#pragma unroll
        for (int q = 0; q < 5; q++) h2[q] = T(p.halo2[q]);
    }
}

// Velocities of plane `pl` (own column, from the shared ring) into the
// reciprocal ring and the division plane with the face-averaged viscosity.
template <typename T, int TJE, bool PPM, bool SST>
__device__ __forceinline__ void plane_prims(Smem<T, TJE, PPM> &s, int pl, int r, int l, T mu_pl, T mu_prev)
{
    constexpr int HW = Smem<T, TJE, PPM>::HW, NS = Smem<T, TJE, PPM>::NS;
    const T *u = s.U[pl & (NS - 1)][r + HW][l + HW];
    vel_rcp(u[0], u[1], u[2], u[3], s.R[pl % 3][r][l]);
    T dv[4];
    vdiv(u, dv);
    T *o = s.Dv[pl & 1][r][l];
    o[0] = dv[0]; o[1] = dv[1]; o[2] = dv[2]; o[3] = dv[3];
    if constexpr (!SST) o[4] = T(0.5) * (mu_pl + mu_prev);
}

// SST: static Smagorinsky (the face viscosity from the face gradients and the
// two cells' densities; no mu field is read).
template <typename T, int TJE, int MINB, bool PPM, bool SST>
__global__ void __launch_bounds__(TJE * 32, MINB) k_stage(Grid g, Consts kc, Args<T> a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    typedef Smem<T, TJE, PPM> SM;
    SM &s = *reinterpret_cast<SM *>(smraw);
    constexpr int HW = SM::HW, NS = SM::NS;
    const int L = g.L, H = g.H, D = g.D;
    constexpr int TJ = TJE - 2;
    const int r = threadIdx.y, l = threadIdx.x;
    const int j = blockIdx.y * TJ + r;
    const int k = blockIdx.x * 30 + l;
    const int i0 = 1 + blockIdx.z * a.seg;
    const int i1 = min(L, i0 + a.seg - 1);
    const bool live = (j <= H + 1) && (k <= D + 1);
    const bool inter = live && r >= 1 && r <= TJE - 2 && l >= 1 && l <= 30 && j <= H && k <= D;
    const bool ycol = live && l >= 1 && l <= 30 && k <= D;     // column takes part in y faces
    const bool zrow = live && r >= 1 && r <= TJE - 2 && j <= H; // row takes part in z faces
    const long long fs = g.fstride;
    const double *__restrict__ cu = a.cur;
    const T *__restrict__ mu = a.mu;
    const long long nxf = (long long)H * D, nyf = (long long)L * D, nzf = (long long)L * H;
    const long long cj = g.idx(0, j, k); // column base (plane 0)

    T hix[5], Fxp[5];
#pragma unroll
    for (int q = 0; q < 5; q++) hix[q] = Fxp[q] = T(0.);
    T mu0 = 0, mu1 = 0, mu2 = 0; // mu of planes i, i+1, i+2 (own column)
    PlaneLoad pl;
#pragma unroll
    for (int q = 0; q < 5; q++) pl.own[q] = pl.halo[q] = pl.halo2[q] = 0.;
    double base[5], unv[5]; // FP64 operands of the stage combination, fetched early
#pragma unroll
    for (int q = 0; q < 5; q++) base[q] = unv[q] = 0.;

    // ---- prologue: planes i0-1 .. i0+1 (PPM: .. i0+2), flux of face i0 - 1/2 ----
    {
        T Um[5] = {0, 0, 0, 0, 0}, mum = 0;
        plane_issue<T, TJE, PPM>(g, cu, i0, r, l, j, k, live, pl);
        plane_store<T, TJE, PPM>(s, i0 & (NS - 1), r, l, j, k, H, D, live, pl);
        plane_issue<T, TJE, PPM>(g, cu, i0 + 1, r, l, j, k, live, pl);
        plane_store<T, TJE, PPM>(s, (i0 + 1) & (NS - 1), r, l, j, k, H, D, live, pl);
        if constexpr (PPM) {
            plane_issue<T, TJE, PPM>(g, cu, i0 + 2, r, l, j, k, live, pl);
            plane_store<T, TJE, PPM>(s, (i0 + 2) & (NS - 1), r, l, j, k, H, D, live && i0 + 2 <= L + 1, pl);
        }
        if (live) {
            load5(cu, fs, cj + (long long)(i0 - 1) * g.pi, Um);
            if constexpr (PPM) {
                // plane i0-1 (own column): the x sweep of cell i0+1 reads it
#pragma unroll
                for (int q = 0; q < 5; q++) s.U[(i0 - 1) & (NS - 1)][r + HW][l + HW][q] = Um[q];
            }
            vel_rcp(Um[0], Um[1], Um[2], Um[3], s.R[(i0 - 1) % 3][r][l]);
            if constexpr (!SST) {
                mum = mu[FSL_CELL(cj + (long long)(i0 - 1) * g.pi, fs)];
                mu0 = mu[FSL_CELL(cj + (long long)i0 * g.pi, fs)];
                mu1 = mu[FSL_CELL(cj + (long long)(i0 + 1) * g.pi, fs)];
            }
            plane_prims<T, TJE, PPM, SST>(s, i0, r, l, mu0, mum);
            plane_prims<T, TJE, PPM, SST>(s, i0 + 1, r, l, mu1, mu0);
        }
        __syncthreads();
        if (inter) {
            T hm[5], lo[5], hin[5], dm[4], tmp[5];
            const T *Uc = s.U[i0 & (NS - 1)][r + HW][l + HW], *Un = s.U[(i0 + 1) & (NS - 1)][r + HW][l + HW];
            {
                CellC<T> cc;
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
                cell_consts(cc);
                if (PPM && i0 >= 2 && i0 <= L - 1) {
                    T m2[5];
                    load5(cu, fs, cj + (long long)(i0 - 2) * g.pi, m2);
                    ppm_x(cc, m2, Um, Un, s.U[(i0 + 2) & (NS - 1)][r + HW][l + HW], hin, lo);
                } else {
                    recon_x(cc, Un, Um, hin, lo);
                }
            }
            if (i0 == 1) {
                const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hm[q] = a.bf.x0[q * nxf + FSL_FACE(fo, nxf)];
            } else if (PPM && i0 - 1 >= 2 && i0 - 1 <= L - 1) {
                ppm_at_x<T>(g, cu, cj + (long long)(i0 - 1) * g.pi, hm, tmp);
            } else {
                recon_at<T, 0>(g, cu, cj + (long long)(i0 - 1) * g.pi, hm, tmp);
            }
            vdiv(Um, dm);
            const T *dc = s.Dv[i0 & 1][r][l];
            const int sb = (i0 - 1) % 3, sf = i0 % 3;
            const T m_f = SST ? T(0.5) * (Uc[0] + Um[0]) : dc[4];
            fused_face<T, 1, SST>(hm, lo, dm, dm[3], dc, dc[3], s.R[sf][r + 1][l], s.R[sb][r + 1][l],
                                  s.R[sf][r - 1][l], s.R[sb][r - 1][l], s.R[sf][r][l + 1], s.R[sb][r][l + 1],
                                  s.R[sf][r][l - 1], s.R[sb][r][l - 1], m_f, kc, Fxp);
#pragma unroll
            for (int q = 0; q < 5; q++) hix[q] = hin[q];
        }
    }
    const double dtx = a.ds->dtx, dty = a.ds->dty, dtz = a.ds->dtz;
    const double one_third = 1. / 3., two_thirds = 2. / 3.;
    // Courant maximum of the cells this thread wrote (with a.co); in shared
    // memory rather than registers, which the FP64 16-row tile has none left of
    __shared__ double comax[TJE][32];
    comax[r][l] = 0.0;
    __syncthreads();

    for (int i = i0; i <= i1; i++) {
        const int sm1 = (i + 2) % 3, s0 = i % 3, sp1 = (i + 1) % 3;
        const int u0 = i & 1, u1 = (i + 1) & 1;                   // Dv ring
        const int q0 = i & (NS - 1), q1 = (i + 1) & (NS - 1);     // state ring: planes i, i+1
        // (a) issue plane i+2 (PPM: i+3) loads (the velocities of plane i+1
        // were formed at the end of the previous iteration, or in the prologue)
        plane_issue<T, TJE, PPM>(g, cu, i + (PPM ? 3 : 2), r, l, j, k, live, pl);
        if (inter) {
            const long long c = FSL_CELL(cj + (long long)i * g.pi, fs);
            // FP32 bulk keeps only a converted copy of the state in shared
            // memory; the FP64 operands of the combination are fetched here
            if (sizeof(T) != 8) {
#pragma unroll
                for (int q = 0; q < 5; q++) base[q] = cu[q * fs + c];
                if (a.stage != 1) {
#pragma unroll
                    for (int q = 0; q < 5; q++) unv[q] = a.un[q * fs + c];
                }
            }
        }
        if (!SST && live && i + 2 <= L + 1) mu2 = mu[FSL_CELL(cj + (long long)(i + 2) * g.pi, fs)];
        // (b) y and z reconstruction of cell (i, j, k): reads the state ring
        // only (plane i, stored two iterations ago)
        T hy[5], hz[5], lz[5];
#pragma unroll
        for (int q = 0; q < 5; q++) hy[q] = hz[q] = lz[q] = T(0.);
        {
            const bool ry = ycol && j >= 1 && j <= H;
            const bool rz = zrow && k >= 1 && k <= D;
            if (ry || rz) {
                CellC<T> cc;
                const T *Uc = s.U[q0][r + HW][l + HW];
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
                cell_consts(cc);
                T fw[5], bw[5], lo[5];
                if (ry) {
                    const T *a1 = s.U[q0][r + HW + 1][l + HW], *b1 = s.U[q0][r + HW - 1][l + HW];
                    fw[0] = a1[0]; fw[1] = a1[2]; fw[2] = a1[3]; fw[3] = a1[1]; fw[4] = a1[4];
                    bw[0] = b1[0]; bw[1] = b1[2]; bw[2] = b1[3]; bw[3] = b1[1]; bw[4] = b1[4];
                    if (PPM && j >= 2 && j <= H - 1) {
                        const T *a2 = s.U[q0][r + HW + 2][l + HW], *b2 = s.U[q0][r + HW - 2][l + HW];
                        T f2[5], b2v[5];
                        f2[0] = a2[0]; f2[1] = a2[2]; f2[2] = a2[3]; f2[3] = a2[1]; f2[4] = a2[4];
                        b2v[0] = b2[0]; b2v[1] = b2[2]; b2v[2] = b2[3]; b2v[3] = b2[1]; b2v[4] = b2[4];
                        ppm_y(cc, b2v, bw, fw, f2, hy, lo);
                    } else {
                        recon_y(cc, fw, bw, hy, lo);
                    }
#pragma unroll
                    for (int q = 0; q < 5; q++) s.Lo[r][l][q] = lo[q];
                }
                if (rz) {
                    const T *a1 = s.U[q0][r + HW][l + HW + 1], *b1 = s.U[q0][r + HW][l + HW - 1];
                    fw[0] = a1[0]; fw[1] = a1[3]; fw[2] = a1[1]; fw[3] = a1[2]; fw[4] = a1[4];
                    bw[0] = b1[0]; bw[1] = b1[3]; bw[2] = b1[1]; bw[3] = b1[2]; bw[4] = b1[4];
                    if (PPM && k >= 2 && k <= D - 1) {
                        const T *a2 = s.U[q0][r + HW][l + HW + 2], *b2 = s.U[q0][r + HW][l + HW - 2];
                        T f2[5], b2v[5];
                        f2[0] = a2[0]; f2[1] = a2[3]; f2[2] = a2[1]; f2[3] = a2[2]; f2[4] = a2[4];
                        b2v[0] = b2[0]; b2v[1] = b2[3]; b2v[2] = b2[1]; b2v[3] = b2[2]; b2v[4] = b2[4];
                        ppm_z(cc, b2v, bw, fw, f2, hz, lz);
                    } else {
                        recon_z(cc, fw, bw, hz, lz);
                    }
                }
            }
            if (ycol && j == 0) {
                const long long fo = (long long)(i - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hy[q] = a.bf.y0[q * nyf + FSL_FACE(fo, nyf)];
            }
            if (ycol && j == H + 1) {
                const long long fo = (long long)(i - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) s.Lo[r][l][q] = a.bf.yH[q * nyf + FSL_FACE(fo, nyf)];
            }
            if (zrow && k == 0) {
                const long long fo = (long long)(i - 1) * H + (j - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hz[q] = a.bf.z0[q * nzf + FSL_FACE(fo, nzf)];
            }
            if (zrow && k == D + 1) {
                const long long fo = (long long)(i - 1) * H + (j - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) lz[q] = a.bf.zD[q * nzf + FSL_FACE(fo, nzf)];
            }
        }
        __syncthreads();
        // (c) y face above the cell: (i, j + 1/2), j in [0, HIG]
        if (ycol && r <= TJE - 2 && j <= H) {
            T F[5];
            const T *vm = s.Dv[u0][r][l], *vp = s.Dv[u0][r + 1][l];
            const T m_f = SST ? T(0.5) * (s.U[q0][r + 1 + HW][l + HW][0] + s.U[q0][r + HW][l + HW][0]) : vp[4];
            fused_face<T, 2, SST>(hy, s.Lo[r + 1][l], vm, vm[3], vp, vp[3], s.R[sp1][r + 1][l], s.R[sp1][r][l],
                                  s.R[sm1][r + 1][l], s.R[sm1][r][l], s.R[s0][r + 1][l + 1], s.R[s0][r][l + 1],
                                  s.R[s0][r + 1][l - 1], s.R[s0][r][l - 1], m_f, kc, F);
#pragma unroll
            for (int q = 0; q < 5; q++) s.Fy[r][l][q] = F[q];
        }
        // (d) z face nearer than the cell: (i, j, k + 1/2), k in [0, DEP]
        T Fz[5], Fzm[5];
        {
            T lzn[5];
#pragma unroll
            for (int q = 0; q < 5; q++) lzn[q] = __shfl_down_sync(0xffffffffu, lz[q], 1);
#pragma unroll
            for (int q = 0; q < 5; q++) Fz[q] = T(0.);
            if (zrow && l <= 30 && k <= D) {
                const T *vm = s.Dv[u0][r][l], *vp = s.Dv[u0][r][l + 1];
                const T m_f = SST ? T(0.5) * (s.U[q0][r + HW][l + 1 + HW][0] + s.U[q0][r + HW][l + HW][0]) : vp[4];
                fused_face<T, 3, SST>(hz, lzn, vm, vm[3], vp, vp[3], s.R[sp1][r][l + 1], s.R[sp1][r][l],
                                      s.R[sm1][r][l + 1], s.R[sm1][r][l], s.R[s0][r + 1][l + 1], s.R[s0][r + 1][l],
                                      s.R[s0][r - 1][l + 1], s.R[s0][r - 1][l], m_f, kc, Fz);
            }
#pragma unroll
            for (int q = 0; q < 5; q++) Fzm[q] = __shfl_up_sync(0xffffffffu, Fz[q], 1);
        }
        // (e) x face (i + 1/2, j, k): reconstruct cell i+1, flux
        T Fx[5], hin[5];
#pragma unroll
        for (int q = 0; q < 5; q++) Fx[q] = hin[q] = T(0.);
        if (inter) {
            T lo[5];
            if (i + 1 <= L) {
                CellC<T> cc;
                const T *Un = s.U[q1][r + HW][l + HW];
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Un[q];
                cell_consts(cc);
                if constexpr (PPM) {
                    // planes i-1 .. i+2 from the ring (own column), i+3 in flight
                    const T *Um1 = s.U[(i - 1) & (NS - 1)][r + HW][l + HW], *U0 = s.U[q0][r + HW][l + HW];
                    const T *Up2 = s.U[(i + 2) & (NS - 1)][r + HW][l + HW];
                    if (i + 1 <= L - 1) {
                        T p2[5];
#pragma unroll
                        for (int q = 0; q < 5; q++) p2[q] = T(pl.own[q]);
                        ppm_x(cc, Um1, U0, Up2, p2, hin, lo);
                    } else {
                        recon_x(cc, Up2, U0, hin, lo);
                    }
                } else {
                    T fw2[5];
#pragma unroll
                    for (int q = 0; q < 5; q++) fw2[q] = T(pl.own[q]);
                    recon_x(cc, fw2, s.U[q0][r + HW][l + HW], hin, lo);
                }
            } else {
                const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) lo[q] = a.bf.xL[q * nxf + FSL_FACE(fo, nxf)];
            }
            const T *dc = s.Dv[u0][r][l], *dn = s.Dv[u1][r][l];
            const T m_f = SST ? T(0.5) * (s.U[q1][r + HW][l + HW][0] + s.U[q0][r + HW][l + HW][0]) : dn[4];
            fused_face<T, 1, SST>(hix, lo, dc, dc[3], dn, dn[3], s.R[sp1][r + 1][l], s.R[s0][r + 1][l],
                                  s.R[sp1][r - 1][l], s.R[s0][r - 1][l], s.R[sp1][r][l + 1], s.R[s0][r][l + 1],
                                  s.R[sp1][r][l - 1], s.R[s0][r][l - 1], m_f, kc, Fx);
        }
        __syncthreads();
        // (f) divergence and stage combination (src/evolution.c:29-161), FP64
        if (inter) {
            const long long c = FSL_CELL(cj + (long long)i * g.pi, fs);
            const T *Uc = s.U[q0][r + HW][l + HW];
            (void)Uc;
#pragma unroll
            for (int q = 0; q < 5; q++) {
                double o;
                if constexpr (sizeof(T) == 8) {
                    // the reference's order, ((b0 + X) + Y) + Z, on the stage
                    // state itself (the shared copy is exact for T = double)
                    const double X = dtx * ((double)Fxp[q] - (double)Fx[q]);
                    const double Y = dty * ((double)s.Fy[r - 1][l][q] - (double)s.Fy[r][l][q]);
                    const double Z = dtz * ((double)Fzm[q] - (double)Fz[q]);
                    const double b0 = (double)Uc[q];
                    if (a.stage != 1) unv[q] = a.un[q * fs + c];
                    if (a.stage == 1) o = b0 + X + Y + Z;
                    else if (a.stage == 2) o = 0.75 * unv[q] + 0.25 * (b0 + X + Y + Z);
                    else o = one_third * unv[q] + two_thirds * (b0 + X + Y + Z);
                } else {
                    // FP32 bulk: the divergence in FP32 (one conversion), the
                    // stage combination in FP64 on the FP64 stage state
                    const T X = T(dtx) * (Fxp[q] - Fx[q]);
                    const T Y = T(dty) * (s.Fy[r - 1][l][q] - s.Fy[r][l][q]);
                    const T Z = T(dtz) * (Fzm[q] - Fz[q]);
                    const double inc = (double)(X + Y + Z);
                    if (a.stage == 1) o = base[q] + inc;
                    else if (a.stage == 2) o = 0.75 * unv[q] + 0.25 * (base[q] + inc);
                    else o = one_third * unv[q] + two_thirds * (base[q] + inc);
                }
                a.out[q * fs + c] = o;
                base[q] = o; // the new state, for the Courant number below
            }
            if (a.co && i >= a.co_i0 && i <= a.co_i1) {
                // the next step's check of src/helpers.c:23-52 on this state
                const double Co = cell_courant(kc.cfl_mode, base[0], base[1], base[2], base[3], base[4], dtx, dty, dtz);
                const double m = comax[r][l];
                comax[r][l] = (Co > m) ? Co : m;
                if (!(base[0] > 0.0)) atomicOr(a.status, 2u);
            }
        }
        // (g) plane i+2 into the ring slot of plane i (all readers of plane i
        // passed the barrier above) and its velocities into the slots of
        // planes i-1 (reciprocal ring) and i (division planes), read next
        // after the next iteration's barrier; advance the march
        if constexpr (PPM)
            plane_store<T, TJE, PPM>(s, (i + 3) & (NS - 1), r, l, j, k, H, D, live && i + 3 <= L + 1, pl);
        else
            plane_store<T, TJE, PPM>(s, q0, r, l, j, k, H, D, live && i + 2 <= L + 1, pl);
        if (live && i < i1) plane_prims<T, TJE, PPM, SST>(s, i + 2, r, l, mu2, mu1);
#pragma unroll
        for (int q = 0; q < 5; q++) {
            Fxp[q] = Fx[q];
            hix[q] = hin[q];
        }
        mu0 = mu1;
        mu1 = mu2;
    }
    if (a.co) {
        __syncthreads();
        double m = comax[r][l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_xor_sync(0xffffffffu, m, o);
            m = (x > m) ? x : m;
        }
        __syncthreads();
        if (l == 0) comax[r][0] = m;
        __syncthreads();
        if (r == 0 && l == 0) {
            m = 0.0;
#pragma unroll
            for (int q = 0; q < TJE; q++) m = (comax[q][0] > m) ? comax[q][0] : m;
            // non-negative doubles order like their bit patterns
            atomicMax(a.co, (unsigned long long)__double_as_longlong(m));
        }
    }
}

template <typename T, int TJE, int MINB, bool PPM = false, bool SST = false>
int launch_stage_t(Ctx &c, int stage, const double *cur, const double *un, double *out, const T *mu, BF<T> bf,
                   bool courant)
{
    const Grid &g = c.g;
    Args<T> a;
    a.cur = cur; a.un = un; a.out = out; a.mu = mu; a.bf = bf; a.ds = c.ds; a.stage = stage;
    a.co = courant ? &c.ds->co_bits : nullptr;
    a.co_i0 = c.co_i0;
    a.co_i1 = c.co_i1;
    a.status = &c.ds->status;
    a.seg = c.stage_seg;
    a.vel = nullptr;
    const size_t smem = sizeof(Smem<T, TJE, PPM>);
    static std::atomic<uint64_t> attr{0};
    if (!smem_limit_once((const void *)k_stage<T, TJE, MINB, PPM, SST>, smem, attr)) return -1;
    dim3 b(32, TJE, 1);
    dim3 gr((g.D + 29) / 30, (g.H + TJE - 3) / (TJE - 2), (g.L + a.seg - 1) / a.seg);
    prof_begin(c, FSL_K_STAGE);
    k_stage<T, TJE, MINB, PPM, SST><<<gr, b, smem, c.stream>>>(g, c.k, a);
    prof_end(c, FSL_K_STAGE, 1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

template <typename T> void launch_bface_t(Ctx &c, const double *cur, const Disturb &d, BF<T> bf)
{
    const Grid &g = c.g;
    const long long n = (long long)g.H * g.D + (long long)g.L * g.D + (long long)g.L * g.H;
    prof_begin(c, FSL_K_BC);
    k_bface<T><<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(g, c.k.setup, c.k.BL_HIG, d, cur, bf);
    prof_end(c, FSL_K_BC, 1);
}

} // namespace stage
} // namespace fsl
