// fsl_fused.cu -- fused RK3 stage: reconstruction, fluxes, divergence and the
// stage combination in one pass over the domain (FP64, --fmad=false).
//
// Decomposition ("2.5-D" streaming): a block owns a tile of (TJE-2) x 30
// cell columns in (y, z) plus a one-cell halo ring (TJE rows = warps, 32
// lanes along the contiguous k axis) and marches along x over `seg` planes.
// Per plane it stages in shared memory the current-stage state (halo 2), the
// two velocity forms the viscous stencil reads (src/fluxes.c divides for the
// two cells adjacent to a face, :117-122, and multiplies by a reciprocal for
// the eight tangential neighbours, :124-142), temperature and the face-averaged
// SGS viscosity.  Every face flux of the tile is computed once (x faces from
// registers carried along the march, y faces through shared memory, z faces
// through warp shuffles); the state is read once and the stage result written
// once.  Domain-boundary faces take their outer state from the boundary pass
// (k_bface), which applies the reference's interface rules
// (src/bounCondOnInterfaces.c:11-110) to the reconstructed boundary cells.
// Every value is formed with the reference's expressions, so the result equals
// the per-phase path (and the reference) bit for bit.
#include "fsl_internal.h"
#include "fsl_phys.cuh"

namespace fsl {

namespace {

__device__ __forceinline__ void load5(const double *__restrict__ u, long long fs, long long c, double *v)
{
#pragma unroll
    for (int q = 0; q < 5; q++) v[q] = u[q * fs + c];
}

// reconstruction sweep DIR (0 x, 1 y, 2 z) of the padded cell c
template <int DIR>
__device__ __forceinline__ void recon_at(const Grid &g, const double *__restrict__ u, long long c, double *hi,
                                         double *lo)
{
    const long long fs = g.fstride;
    CellC<double> cc;
    load5(u, fs, c, cc.u);
    cell_consts(cc);
    const long long d = DIR == 0 ? g.pi : DIR == 1 ? (long long)g.pk : 1LL;
    const int p1 = DIR == 0 ? 1 : DIR == 1 ? 2 : 3;
    const int p2 = DIR == 0 ? 2 : DIR == 1 ? 3 : 1;
    const int p3 = DIR == 0 ? 3 : DIR == 1 ? 1 : 2;
    double fw[5], bw[5];
    fw[0] = u[c + d]; fw[1] = u[p1 * fs + c + d]; fw[2] = u[p2 * fs + c + d]; fw[3] = u[p3 * fs + c + d];
    fw[4] = u[4 * fs + c + d];
    bw[0] = u[c - d]; bw[1] = u[p1 * fs + c - d]; bw[2] = u[p2 * fs + c - d]; bw[3] = u[p3 * fs + c - d];
    bw[4] = u[4 * fs + c - d];
    if (DIR == 0) recon_x(cc, fw, bw, hi, lo);
    else if (DIR == 1) recon_y(cc, fw, bw, hi, lo);
    else recon_z(cc, fw, bw, hi, lo);
}

// Outer states of all domain-boundary faces (src/bounCondOnInterfaces.c:11-110).
__global__ void k_bface(Grid g, int setup, int BL_HIG, Disturb d, const double *__restrict__ u, BFaces bf)
{
    const int L = g.L, H = g.H, D = g.D;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nx = (long long)H * D, ny = (long long)L * D, nz = (long long)L * H;
    const bool spatial = (setup == FSL_SETUP_SPATIAL);
    typedef Kc<double> kc;
    double hi[5], lo[5];
    if (t < nx) {
        const int jf = (int)(t / D), kf = (int)(t % D);
        const int j = jf + 1, k = kf + 1;
        const long long fo = t;
        if (spatial) {
            const double P = 100000., R = 1.0;
            double U, V = 0., W = 0., v[5];
            if (jf < H / 2) { // :17-29
                U = 76.4;
                v[0] = R; v[1] = R * U; v[2] = 0.; v[3] = 0.; v[4] = P / kc::K_1 + 0.5 * R * (U * U);
            } else if (jf < H / 2 + BL_HIG) { // :31-49
                const unsigned ku = (unsigned)kf;
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
            for (int q = 0; q < 5; q++) bf.x0[q * nx + fo] = v[q];
            // :62-71 outflow from the minus state of face LEN
            recon_at<0>(g, u, g.idx(L, j, k), hi, lo);
            const double r = hi[0], mu_ = hi[1], mv = hi[2], mw = hi[3];
            bf.xL[fo] = r; bf.xL[nx + fo] = mu_; bf.xL[2 * nx + fo] = mv; bf.xL[3 * nx + fo] = mw;
            bf.xL[4 * nx + fo] = P / kc::K_1 + 0.5 * (mu_ * mu_ + mv * mv + mw * mw) / r;
        } else { // periodic x, the reference's z rule (:94-109)
            recon_at<0>(g, u, g.idx(L, j, k), hi, lo);
#pragma unroll
            for (int q = 0; q < 5; q++) bf.x0[q * nx + fo] = hi[q];
            recon_at<0>(g, u, g.idx(1, j, k), hi, lo);
#pragma unroll
            for (int q = 0; q < 5; q++) bf.xL[q * nx + fo] = lo[q];
        }
    } else if ((t -= nx) < ny) { // :75-90
        const int i = (int)(t / D) + 1, k = (int)(t % D) + 1;
        recon_at<1>(g, u, g.idx(i, 1, k), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.y0[q * ny + t] = (q == 2 && spatial) ? -lo[q] : lo[q];
        recon_at<1>(g, u, g.idx(i, H, k), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.yH[q * ny + t] = (q == 2 && spatial) ? -hi[q] : hi[q];
    } else if ((t -= ny) < nz) { // :94-109
        const int i = (int)(t / H) + 1, j = (int)(t % H) + 1;
        recon_at<2>(g, u, g.idx(i, j, D), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.z0[q * nz + t] = hi[q];
        recon_at<2>(g, u, g.idx(i, j, 1), hi, lo);
#pragma unroll
        for (int q = 0; q < 5; q++) bf.zD[q * nz + t] = lo[q];
    }
}

template <int TJE> struct StageSmem {
    double U[TJE + 2][34][5]; // current-stage state at plane i, halo 2
    double R[3][TJE][32][3];  // velocities by reciprocal, planes i-1, i, i+1 (ring)
    double Dv[TJE][32][5];    // velocities by division, temperature, mu face average, plane i
    double Lo[TJE][32][5];    // y sweep: state on the face below each cell
    double Fy[TJE][32][5];    // y flux on the face above each row
};

struct StageArgs {
    const double *cur; // current-stage state, ghost layer filled
    const double *un;  // U^n
    double *out;
    const double *mu;
    BFaces bf;
    const DevScalars *ds;
    int stage;
    int seg;
};

// Flux of one face (src/fluxes.c): Riemann state from the two face states,
// viscous and heat flux from the two adjacent cells (vm/Tm minus side, vp/Tp
// plus side, by division) and the eight tangential neighbours (by
// reciprocal; P/M = plus/minus cell, h/l = +/- along the first (1) and
// second (2) tangential axis).
template <int N>
__device__ __forceinline__ void fused_face(const double *Lm, const double *Rp, const double *vm, double Tm,
                                           const double *vp, double Tp, const double *Ph1, const double *Mh1,
                                           const double *Pl1, const double *Ml1, const double *Ph2,
                                           const double *Mh2, const double *Pl2, const double *Ml2, double muT,
                                           const Consts &kc, double *F)
{
    double Rho, P, vel[3];
    riemann<double, N>(Lm, Rp, Rho, P, vel);
    const int n0 = N - 1;
    const int t1 = (N == 1) ? 1 : 0;
    const int t2 = (N == 3) ? 1 : 2;
    const double rdn = N == 1 ? kc.rdx : N == 2 ? kc.rdy : kc.rdz;
    const double rt1 = N == 1 ? kc.r4dy : kc.r4dx;
    const double rt2 = N == 3 ? kc.r4dy : kc.r4dz;
    double gr[3][3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        gr[q][n0] = (vp[q] - vm[q]) * rdn;
        gr[q][t1] = (Ph1[q] + Mh1[q] - Pl1[q] - Ml1[q]) * rt1;
        gr[q][t2] = (Ph2[q] + Mh2[q] - Pl2[q] - Ml2[q]) * rt2;
    }
    face_flux<double, N>(Rho, P, vel, gr, vp, vm, Tp, Tm, kc.mu_L, muT, kc.lambda_L, kc.cp_Pr_T, rdn, F);
}

__device__ __forceinline__ void vdiv(const double *U, double *o)
{
    double Tt;
    vel_div(U[0], U[1], U[2], U[3], U[4], o, Tt);
    o[3] = Tt;
}

template <int TJE>
__global__ void __launch_bounds__(TJE * 32, 1) k_stage(Grid g, Consts kc, StageArgs a)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    StageSmem<TJE> &s = *reinterpret_cast<StageSmem<TJE> *>(smraw);
    const int L = g.L, H = g.H, D = g.D;
    constexpr int TJ = TJE - 2;
    const int r = threadIdx.y, l = threadIdx.x;
    const int j = blockIdx.y * TJ + r;
    const int k = blockIdx.x * 30 + l;
    const int i0 = 1 + blockIdx.z * a.seg;
    const int i1 = min(L, i0 + a.seg - 1);
    const bool live = (j <= H + 1) && (k <= D + 1);
    const bool inter = live && r >= 1 && r <= TJE - 2 && l >= 1 && l <= 30 && j <= H && k <= D;
    const bool ycol = live && l >= 1 && l <= 30 && k <= D;          // column takes part in y faces
    const bool zrow = live && r >= 1 && r <= TJE - 2 && j <= H;      // row takes part in z faces
    const long long fs = g.fstride;
    const double *__restrict__ cu = a.cur;
    const double *__restrict__ mu = a.mu;
    const long long nxf = (long long)H * D, nyf = (long long)L * D, nzf = (long long)L * H;

    double Uc[5], Un1[5], Un2[5], dc[4], dn[4];
    double mum = 0, muc = 0, mun = 0;
    double hix[5], Fxp[5];
#pragma unroll
    for (int q = 0; q < 5; q++) { Uc[q] = Un1[q] = Un2[q] = hix[q] = Fxp[q] = 0.; }
#pragma unroll
    for (int q = 0; q < 4; q++) dc[q] = dn[q] = 0.;

    // ---- prologue: planes i0-1 and i0, flux of face i0 - 1/2 ----
    double Um[5] = {0, 0, 0, 0, 0}, dm[4] = {0, 0, 0, 0};
    if (live) {
        const long long c = g.idx(i0, j, k);
        load5(cu, fs, c - g.pi, Um);
        load5(cu, fs, c, Uc);
        load5(cu, fs, c + g.pi, Un1);
        vel_rcp(Um[0], Um[1], Um[2], Um[3], s.R[(i0 - 1) % 3][r][l]);
        vel_rcp(Uc[0], Uc[1], Uc[2], Uc[3], s.R[i0 % 3][r][l]);
        vdiv(Um, dm);
        vdiv(Uc, dc);
        mum = mu[c - g.pi];
        muc = mu[c];
    }
    __syncthreads();
    if (inter) {
        double hm[5], lo[5], hin[5], tmp[5];
        {
            CellC<double> cc;
#pragma unroll
            for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
            cell_consts(cc);
            recon_x(cc, Un1, Um, hin, lo);
        }
        if (i0 == 1) {
            const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
            for (int q = 0; q < 5; q++) hm[q] = a.bf.x0[q * nxf + fo];
        } else {
            recon_at<0>(g, cu, g.idx(i0 - 1, j, k), hm, tmp);
        }
        const int sb = (i0 - 1) % 3, sf = i0 % 3;
        fused_face<1>(hm, lo, dm, dm[3], dc, dc[3], s.R[sf][r + 1][l], s.R[sb][r + 1][l], s.R[sf][r - 1][l],
                      s.R[sb][r - 1][l], s.R[sf][r][l + 1], s.R[sb][r][l + 1], s.R[sf][r][l - 1],
                      s.R[sb][r][l - 1], 0.5 * (muc + mum), kc, Fxp);
#pragma unroll
        for (int q = 0; q < 5; q++) hix[q] = hin[q];
    }
    const double dtx = a.ds->dtx, dty = a.ds->dty, dtz = a.ds->dtz;
    const double one_third = 1. / 3., two_thirds = 2. / 3.;
    __syncthreads();

    for (int i = i0; i <= i1; i++) {
        const int sm1 = (i + 2) % 3, s0 = i % 3, sp1 = (i + 1) % 3;
        // (a) stage plane i, prepare plane i+1
        if (live) {
            const long long c = g.idx(i, j, k);
            if (i + 2 <= L + 1) load5(cu, fs, c + 2 * g.pi, Un2);
            mun = mu[c + g.pi];
            vel_rcp(Un1[0], Un1[1], Un1[2], Un1[3], s.R[sp1][r][l]);
            vdiv(Un1, dn);
            s.Dv[r][l][0] = dc[0]; s.Dv[r][l][1] = dc[1]; s.Dv[r][l][2] = dc[2]; s.Dv[r][l][3] = dc[3];
            s.Dv[r][l][4] = 0.5 * (muc + mum);
#pragma unroll
            for (int q = 0; q < 5; q++) s.U[r + 1][l + 1][q] = Uc[q];
            if (r == 0 && j >= 1) load5(cu, fs, c - g.pk, s.U[0][l + 1]);
            if (r == TJE - 1 && j <= H) load5(cu, fs, c + g.pk, s.U[TJE + 1][l + 1]);
            if (l == 0 && k >= 1) load5(cu, fs, c - 1, s.U[r + 1][0]);
            if (l == 31 && k <= D) load5(cu, fs, c + 1, s.U[r + 1][33]);
        }
        __syncthreads();
        // (b) y and z reconstruction of cell (i, j, k)
        double hy[5], hz[5], lz[5];
#pragma unroll
        for (int q = 0; q < 5; q++) hy[q] = hz[q] = lz[q] = 0.;
        {
            const bool ry = ycol && j >= 1 && j <= H;
            const bool rz = zrow && k >= 1 && k <= D;
            if (ry || rz) {
                CellC<double> cc;
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
                cell_consts(cc);
                double fw[5], bw[5], lo[5];
                if (ry) {
                    const double *a1 = s.U[r + 2][l + 1], *b1 = s.U[r][l + 1];
                    fw[0] = a1[0]; fw[1] = a1[2]; fw[2] = a1[3]; fw[3] = a1[1]; fw[4] = a1[4];
                    bw[0] = b1[0]; bw[1] = b1[2]; bw[2] = b1[3]; bw[3] = b1[1]; bw[4] = b1[4];
                    recon_y(cc, fw, bw, hy, lo);
#pragma unroll
                    for (int q = 0; q < 5; q++) s.Lo[r][l][q] = lo[q];
                }
                if (rz) {
                    const double *a1 = s.U[r + 1][l + 2], *b1 = s.U[r + 1][l];
                    fw[0] = a1[0]; fw[1] = a1[3]; fw[2] = a1[1]; fw[3] = a1[2]; fw[4] = a1[4];
                    bw[0] = b1[0]; bw[1] = b1[3]; bw[2] = b1[1]; bw[3] = b1[2]; bw[4] = b1[4];
                    recon_z(cc, fw, bw, hz, lz);
                }
            }
            if (ycol && j == 0) {
                const long long fo = (long long)(i - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hy[q] = a.bf.y0[q * nyf + fo];
            }
            if (ycol && j == H + 1) {
                const long long fo = (long long)(i - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) s.Lo[r][l][q] = a.bf.yH[q * nyf + fo];
            }
            if (zrow && k == 0) {
                const long long fo = (long long)(i - 1) * H + (j - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hz[q] = a.bf.z0[q * nzf + fo];
            }
            if (zrow && k == D + 1) {
                const long long fo = (long long)(i - 1) * H + (j - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) lz[q] = a.bf.zD[q * nzf + fo];
            }
        }
        __syncthreads();
        // (c) y face above the cell: (i, j + 1/2), j in [0, HIG]
        if (ycol && r <= TJE - 2 && j <= H) {
            double F[5];
            const double *vm = s.Dv[r][l], *vp = s.Dv[r + 1][l];
            fused_face<2>(hy, s.Lo[r + 1][l], vm, vm[3], vp, vp[3], s.R[sp1][r + 1][l], s.R[sp1][r][l],
                          s.R[sm1][r + 1][l], s.R[sm1][r][l], s.R[s0][r + 1][l + 1], s.R[s0][r][l + 1],
                          s.R[s0][r + 1][l - 1], s.R[s0][r][l - 1], vp[4], kc, F);
#pragma unroll
            for (int q = 0; q < 5; q++) s.Fy[r][l][q] = F[q];
        }
        // (d) z face nearer than the cell: (i, j, k + 1/2), k in [0, DEP]
        double Fz[5], Fzm[5];
        {
            double lzn[5];
#pragma unroll
            for (int q = 0; q < 5; q++) lzn[q] = __shfl_down_sync(0xffffffffu, lz[q], 1);
#pragma unroll
            for (int q = 0; q < 5; q++) Fz[q] = 0.;
            if (zrow && l <= 30 && k <= D) {
                const double *vm = s.Dv[r][l], *vp = s.Dv[r][l + 1];
                fused_face<3>(hz, lzn, vm, vm[3], vp, vp[3], s.R[sp1][r][l + 1], s.R[sp1][r][l],
                              s.R[sm1][r][l + 1], s.R[sm1][r][l], s.R[s0][r + 1][l + 1], s.R[s0][r + 1][l],
                              s.R[s0][r - 1][l + 1], s.R[s0][r - 1][l], vp[4], kc, Fz);
            }
#pragma unroll
            for (int q = 0; q < 5; q++) Fzm[q] = __shfl_up_sync(0xffffffffu, Fz[q], 1);
        }
        // (e) x face (i + 1/2, j, k): reconstruct cell i+1, flux
        double Fx[5], hin[5];
#pragma unroll
        for (int q = 0; q < 5; q++) Fx[q] = hin[q] = 0.;
        if (inter) {
            double lo[5];
            if (i + 1 <= L) {
                CellC<double> cc;
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Un1[q];
                cell_consts(cc);
                recon_x(cc, Un2, Uc, hin, lo);
            } else {
                const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) lo[q] = a.bf.xL[q * nxf + fo];
            }
            fused_face<1>(hix, lo, dc, dc[3], dn, dn[3], s.R[sp1][r + 1][l], s.R[s0][r + 1][l],
                          s.R[sp1][r - 1][l], s.R[s0][r - 1][l], s.R[sp1][r][l + 1], s.R[s0][r][l + 1],
                          s.R[sp1][r][l - 1], s.R[s0][r][l - 1], 0.5 * (mun + muc), kc, Fx);
        }
        __syncthreads();
        // (f) divergence and stage combination (src/evolution.c:29-161)
        if (inter) {
            const long long c = g.idx(i, j, k);
#pragma unroll
            for (int q = 0; q < 5; q++) {
                const double X = dtx * (Fxp[q] - Fx[q]);
                const double Y = dty * (s.Fy[r - 1][l][q] - s.Fy[r][l][q]);
                const double Z = dtz * (Fzm[q] - Fz[q]);
                double o;
                if (a.stage == 1) o = Uc[q] + X + Y + Z;
                else if (a.stage == 2) o = 0.75 * a.un[q * fs + c] + 0.25 * (Uc[q] + X + Y + Z);
                else o = one_third * a.un[q * fs + c] + two_thirds * (Uc[q] + X + Y + Z);
                a.out[q * fs + c] = o;
            }
        }
        // (g) advance the march
#pragma unroll
        for (int q = 0; q < 5; q++) {
            Fxp[q] = Fx[q];
            hix[q] = hin[q];
            Uc[q] = Un1[q];
            Un1[q] = Un2[q];
        }
#pragma unroll
        for (int q = 0; q < 4; q++) dc[q] = dn[q];
        mum = muc;
        muc = mun;
        __syncthreads();
    }
}

template <int TJE> int launch_stage_t(Ctx &c, int stage, const double *cur, const double *un, double *out)
{
    const Grid &g = c.g;
    StageArgs a;
    a.cur = cur; a.un = un; a.out = out; a.mu = c.mu; a.bf = c.bf; a.ds = c.ds; a.stage = stage;
    a.seg = c.stage_seg;
    const size_t smem = sizeof(StageSmem<TJE>);
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_stage<TJE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess)
            return -1;
        attr = true;
    }
    dim3 b(32, TJE, 1);
    dim3 gr((g.D + 29) / 30, (g.H + TJE - 3) / (TJE - 2), (g.L + a.seg - 1) / a.seg);
    prof_begin(c, FSL_K_STAGE);
    k_stage<TJE><<<gr, b, smem, c.stream>>>(g, c.k, a);
    prof_end(c, FSL_K_STAGE, 1);
    return 0;
}

} // namespace

void launch_bface(Ctx &c, const double *cur, const Disturb &d)
{
    const Grid &g = c.g;
    const long long n = (long long)g.H * g.D + (long long)g.L * g.D + (long long)g.L * g.H;
    prof_begin(c, FSL_K_BC);
    k_bface<<<(unsigned)((n + 127) / 128), 128, 0, c.stream>>>(g, c.k.setup, c.k.BL_HIG, d, cur, c.bf);
    prof_end(c, FSL_K_BC, 1);
}

int launch_stage(Ctx &c, int stage, const double *cur, const double *un, double *out)
{
    switch (c.stage_tje) {
    case 8: return launch_stage_t<8>(c, stage, cur, un, out);
    case 16: return launch_stage_t<16>(c, stage, cur, un, out);
    default: return launch_stage_t<12>(c, stage, cur, un, out);
    }
}

} // namespace fsl
