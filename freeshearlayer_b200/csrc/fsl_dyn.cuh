// fsl_dyn.cuh -- the dynamic Smagorinsky procedure (src/turbulence.c:17-507)
// as seven passes, templated on the arithmetic type T: T = double in
// fsl_phase.cu (the plain method, compiled with --fmad=false, bit-identical to
// the reference) and T = float in fsl_dyn32.cu (the FP32-bulk path's
// filtering and coefficient).  The conserved state U stays FP64 in both.
#pragma once

#include "fsl_check.cuh"
#include "fsl_internal.h"

namespace fsl {
namespace dyn {

constexpr double H3 = 1. / 3.; // box test-filter weight, src/turbulence.c:113

// ---------------------------------------------------------------------------
// A5/A6 (src/turbulence.c:17-507).
// The filter keeps the reference's three sweeps (y, z, x), each
// t = 0; t += a h; t += b h; t += c h, on zero-initialised scratch whose never
// written bands stay zero (the oracle convention for src/turbulence.c:44-45).
// ---------------------------------------------------------------------------
template <typename T> __global__ void k_dyn_vel(Grid g, const double *__restrict__ U, T *__restrict__ vel)
{
    const long long n = (long long)(g.L + 2) * g.pi;
    const long long fs = g.fstride;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
         t += (long long)gridDim.x * blockDim.x) {
        const long long c = FSL_CELL(g.off + t, fs);
        const T rr = T(1.) / T(U[c]); // :201-205
        vel[c] = T(U[fs + c]) * rr;
        vel[fs + c] = T(U[2 * fs + c]) * rr;
        vel[2 * fs + c] = T(U[3 * fs + c]) * rr;
    }
}

// y sweep (:47-61) of u, v, w and their six products (:213-230), computed
// on the fly; i in [0,LEN], j in [1,HIG], k in [0,DEP].
template <typename T> __global__ void k_filt_y_vel(Grid g, const T *__restrict__ vel, T *__restrict__ t1)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -(long long)g.pk, (long long)g.pk, fs)) return;
    T a[3][3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const long long s = c + (r - 1) * (long long)g.pk;
        a[r][0] = vel[s]; a[r][1] = vel[fs + s]; a[r][2] = vel[2 * fs + s];
    }
    T q[3][9];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        const T uu = a[r][0], vv = a[r][1], ww = a[r][2];
        q[r][0] = uu; q[r][1] = vv; q[r][2] = ww;
        q[r][3] = uu * uu; q[r][4] = uu * vv; q[r][5] = uu * ww;
        q[r][6] = vv * vv; q[r][7] = vv * ww; q[r][8] = ww * ww;
    }
#pragma unroll
    for (int m = 0; m < 9; m++) {
        T t = 0.;
        t += q[0][m] * T(H3); t += q[1][m] * T(H3); t += q[2][m] * T(H3);
        t1[m * fs + c] = t;
    }
}

// generic y sweep of nf fields
template <typename T> __global__ void k_filt_y(Grid g, int nf, const T *__restrict__ src, T *__restrict__ t1)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -(long long)g.pk, (long long)g.pk, fs)) return;
    for (int m = 0; m < nf; m++) {
        const T *s = src + m * fs;
        T t = 0.;
        t += s[c - g.pk] * T(H3); t += s[c] * T(H3); t += s[c + g.pk] * T(H3);
        t1[m * fs + c] = t;
    }
}

// z sweep (:63-77): i in [0,LEN], j in [0,HIG], k in [1,DEP]
template <typename T> __global__ void k_filt_z(Grid g, int nf, const T *__restrict__ t1, T *__restrict__ t2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -1LL, 1LL, fs)) return;
    for (int m = 0; m < nf; m++) {
        const T *s = t1 + m * fs;
        T t = 0.;
        t += s[c - 1] * T(H3); t += s[c] * T(H3); t += s[c + 1] * T(H3);
        t2[m * fs + c] = t;
    }
}

// x sweep (:80-95) back into the pass-1 buffer: i in [1,LEN], j in [0,HIG],
// k in [0,DEP]
template <typename T> __global__ void k_filt_x(Grid g, int nf, const T *__restrict__ t2, T *__restrict__ t1)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z + 1;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -g.pi, g.pi, fs)) return;
    for (int m = 0; m < nf; m++) {
        const T *s = t2 + m * fs;
        T t = 0.;
        t += s[c - g.pi] * T(H3); t += s[c] * T(H3); t += s[c + g.pi] * T(H3);
        t1[m * fs + c] = t;
    }
}

// Interior: Leonard stress, |S|, A_ij = |S| S_ij, B_ij = |S^| S^_ij
// (:250-382).  Field order of the symmetric tensors: 11 12 13 22 23 33.
template <typename T>
__global__ void k_dyn_mid(Grid g, Consts kc, const T *__restrict__ vel, const T *__restrict__ F, T *__restrict__ Lst,
                          T *__restrict__ A, T *__restrict__ B, T *__restrict__ Smag)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -g.pi, g.pi, fs)) return;
    const T f0 = F[c], f1 = F[fs + c], f2 = F[2 * fs + c];
    Lst[c] = F[3 * fs + c] - f0 * f0;
    Lst[fs + c] = F[4 * fs + c] - f0 * f1;
    Lst[2 * fs + c] = F[5 * fs + c] - f0 * f2;
    Lst[3 * fs + c] = F[6 * fs + c] - f1 * f1;
    Lst[4 * fs + c] = F[7 * fs + c] - f1 * f2;
    Lst[5 * fs + c] = F[8 * fs + c] - f2 * f2;
    const long long dI = g.pi, dJ = g.pk;
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
        const T *uu = pass ? F : vel;
        const T *vv = uu + fs, *ww = uu + 2 * fs;
        const T du_dx = (uu[c + dI] - uu[c - dI]) * T(kc.r2dx);
        const T du_dy = (uu[c + dJ] - uu[c - dJ]) * T(kc.r2dy);
        const T du_dz = (uu[c + 1] - uu[c - 1]) * T(kc.r2dz);
        const T dv_dx = (vv[c + dI] - vv[c - dI]) * T(kc.r2dx);
        const T dv_dy = (vv[c + dJ] - vv[c - dJ]) * T(kc.r2dy);
        const T dv_dz = (vv[c + 1] - vv[c - 1]) * T(kc.r2dz);
        const T dw_dx = (ww[c + dI] - ww[c - dI]) * T(kc.r2dx);
        const T dw_dy = (ww[c + dJ] - ww[c - dJ]) * T(kc.r2dy);
        const T dw_dz = (ww[c + 1] - ww[c - 1]) * T(kc.r2dz);
        const T S11 = du_dx, S12 = 0.5 * (du_dy + dv_dx), S13 = 0.5 * (du_dz + dw_dx);
        const T S21 = S12, S22 = dv_dy, S23 = 0.5 * (dv_dz + dw_dy);
        const T S31 = S13, S32 = S23, S33 = dw_dz;
        const T S = sqrt(2 * (S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 +
                                   S31 * S31 + S32 * S32 + S33 * S33));
        T *o = pass ? B : A;
        o[c] = S * S11; o[fs + c] = S * S12; o[2 * fs + c] = S * S13;
        o[3 * fs + c] = S * S22; o[4 * fs + c] = S * S23; o[5 * fs + c] = S * S33;
        if (!pass) Smag[c] = S;
    }
}

// M_ij, Germano-Lilly coefficient with clipping to [0, 0.15], mu_SGS
// (:398-445).
template <typename T>
__global__ void k_dyn_final(Grid g, Consts kc, const double *__restrict__ rho, const T *__restrict__ Lst,
                            const T *__restrict__ B, const T *__restrict__ Ahat, const T *__restrict__ Smag,
                            T *__restrict__ mu, float *__restrict__ cd)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, 0LL, 0LL, fs)) return;
    const T DD = T(kc.DD);
    const T M11 = DD * (4 * B[c] - Ahat[c]);
    const T M12 = DD * (4 * B[fs + c] - Ahat[fs + c]);
    const T M13 = DD * (4 * B[2 * fs + c] - Ahat[2 * fs + c]);
    const T M22 = DD * (4 * B[3 * fs + c] - Ahat[3 * fs + c]);
    const T M23 = DD * (4 * B[4 * fs + c] - Ahat[4 * fs + c]);
    const T M33 = DD * (4 * B[5 * fs + c] - Ahat[5 * fs + c]);
    T L11 = Lst[c], L12 = Lst[fs + c], L13 = Lst[2 * fs + c];
    T L22 = Lst[3 * fs + c], L23 = Lst[4 * fs + c], L33 = Lst[5 * fs + c];
    const T tr = -(1.0 / 3.0) * (L11 + L22 + L33);
    L11 += tr; L22 += tr; L33 += tr;
    const T LLMM = (L11 * M11 + L12 * M12 + L13 * M13 + L12 * M12 + L22 * M22 + L23 * M23 +
                         L13 * M13 + L23 * M23 + L33 * M33);
    const T MMMM = (M11 * M11 + M12 * M12 + M13 * M13 + M12 * M12 + M22 * M22 + M23 * M23 +
                         M13 * M13 + M23 * M23 + M33 * M33);
    T Cd = -0.5 * (LLMM / (MMMM + 1e-30));
    if (Cd > 0.15) Cd = 0.15;
    else if (Cd < 0.0) Cd = 0.0;
    mu[c] = T(rho[c]) * Cd * DD * Smag[c];
    if (cd) cd[c] = (float)Cd; // Cs^2 for the learned closure's harvest and judgement
}


// ---------------------------------------------------------------------------
// Fused evaluation: the same arithmetic in three streaming kernels.
//
// k_dyn_filter9 marches along x over a (TJ rows x 32 k) tile of output
// positions: per plane it stages the velocities (halo 1 in y and z) in shared
// memory, forms the y pass of u, v, w and their six products, the z pass per
// own position, and the x pass from the last three z-pass planes it keeps in
// registers -- each sum as t = 0; t += a h; t += b h; t += c h, on the
// reference's write regions (pass 1: i in [0,L], j in [1,H], k in [0,D];
// pass 2: k in [1,D]; pass 3: i in [1,L]; plane 0 keeps the y-pass value,
// src/turbulence.c:44-95).  Positions outside those regions are never
// written and stay zero, so the output equals the seven-pass result
// everywhere.  k_dyn_strain forms A = |S| S and |S| of the interior
// (src/turbulence.c:273-311).  k_dyn_filterA_final filters A the same way
// (A is zero outside the interior, where the zero bands and a plain filter
// agree) and, per interior cell, forms the Leonard stress, |S^| S^ from the
// filtered velocities, M, the clipped coefficient and mu_SGS
// (src/turbulence.c:250-445) without storing L or B.
// ---------------------------------------------------------------------------
template <typename T> struct Scratch3 {
    T *vel; // 3 fields
    T *F;   // 9 fields, zero outside the filter's write regions (never written there)
    T *A;   // 6 fields, zero on the ghost layer (never written there)
    T *S;   // |S| of the interior
};

template <typename T, int TJ>
__global__ void __launch_bounds__(32 * TJ) k_dyn_filter9(Grid g, int seg, const T *__restrict__ vel, T *__restrict__ F)
{
    __shared__ T vq[TJ + 2][34][3];
    __shared__ T t1[TJ][34][9];
    const int L = g.L, H = g.H, D = g.D;
    const int l = threadIdx.x, r = threadIdx.y, tid = r * 32 + l, nt = 32 * TJ;
    const int k0 = blockIdx.x * 32, j0 = 1 + blockIdx.y * TJ;
    const int j = j0 + r, k = k0 + l;
    const int i0 = blockIdx.z * seg, i1 = min(L, i0 + seg - 1);
    const long long fs = g.fstride;
    const bool own = j <= H && k <= D;
    T p2[9], p1[9], cur[9];
#pragma unroll
    for (int m = 0; m < 9; m++) p2[m] = p1[m] = cur[m] = T(0.);
    const int ib = max(i0 - 1, 0), ie = min(i1 + 1, L + 1);
    // the staged region (TJ+2) x 34 of a plane, at most two positions per
    // thread; plane ip+1 is loaded into registers while plane ip is filtered
    constexpr int NP = ((TJ + 2) * 34 + 32 * TJ - 1) / (32 * TJ);
    T pre[NP][3];
    auto issue = [&](int ip) {
#pragma unroll
        for (int s = 0; s < NP; s++) {
            const int e = tid + s * nt;
            const int rr = e / 34, cc = e % 34, jj = j0 - 1 + rr, kk = k0 - 1 + cc;
            pre[s][0] = pre[s][1] = pre[s][2] = T(0.);
            if (e < (TJ + 2) * 34 && ip <= L && jj <= H + 1 && kk >= 0 && kk <= D + 1) {
                const long long q = FSL_CELL(g.idx(ip, jj, kk), fs);
                pre[s][0] = vel[q]; pre[s][1] = vel[fs + q]; pre[s][2] = vel[2 * fs + q];
            }
        }
    };
    issue(ib);
    for (int ip = ib; ip <= ie; ip++) {
        if (ip <= L) {
#pragma unroll
            for (int s = 0; s < NP; s++) {
                const int e = tid + s * nt;
                if (e < (TJ + 2) * 34) {
                    const int rr = e / 34, cc = e % 34;
                    vq[rr][cc][0] = pre[s][0]; vq[rr][cc][1] = pre[s][1]; vq[rr][cc][2] = pre[s][2];
                }
            }
            issue(ip + 1);
            __syncthreads();
            // pass 1 (y) of the nine fields at rows j0.., columns k0-1 .. k0+32
            for (int e = tid; e < TJ * 34; e += nt) {
                const int rr = e / 34, cc = e % 34, jj = j0 + rr, kk = k0 - 1 + cc;
                T o[9];
                if (jj <= H && kk >= 0 && kk <= D) {
                    T q[3][9];
#pragma unroll
                    for (int w = 0; w < 3; w++) {
                        const T uu = vq[rr + w][cc][0], vv = vq[rr + w][cc][1], ww = vq[rr + w][cc][2];
                        q[w][0] = uu; q[w][1] = vv; q[w][2] = ww;
                        q[w][3] = uu * uu; q[w][4] = uu * vv; q[w][5] = uu * ww;
                        q[w][6] = vv * vv; q[w][7] = vv * ww; q[w][8] = ww * ww;
                    }
#pragma unroll
                    for (int m = 0; m < 9; m++) {
                        T t = 0.;
                        t += q[0][m] * T(H3); t += q[1][m] * T(H3); t += q[2][m] * T(H3);
                        o[m] = t;
                    }
                } else {
#pragma unroll
                    for (int m = 0; m < 9; m++) o[m] = T(0.);
                }
#pragma unroll
                for (int m = 0; m < 9; m++) t1[rr][cc][m] = o[m];
            }
            __syncthreads();
            // pass 2 (z) at the own position
            if (own && k >= 1) {
#pragma unroll
                for (int m = 0; m < 9; m++) {
                    T t = 0.;
                    t += t1[r][l][m] * T(H3); t += t1[r][l + 1][m] * T(H3); t += t1[r][l + 2][m] * T(H3);
                    cur[m] = t;
                }
            } else {
#pragma unroll
                for (int m = 0; m < 9; m++) cur[m] = T(0.);
            }
            // plane 0 keeps its pass-1 value
            if (ip == 0 && own) {
                const long long c = FSL_CELL(g.idx(0, j, k), fs);
#pragma unroll
                for (int m = 0; m < 9; m++) F[m * fs + c] = t1[r][l + 1][m];
            }
            __syncthreads(); // the next plane overwrites vq and t1
        } else {
#pragma unroll
            for (int m = 0; m < 9; m++) cur[m] = T(0.); // plane L+1: pass 2 writes nothing there
        }
        // pass 3 (x) of plane ip-1
        const int io = ip - 1;
        if (io >= max(i0, 1) && io <= i1 && own && k >= 1) {
            const long long c = FSL_CELL(g.idx(io, j, k), fs);
#pragma unroll
            for (int m = 0; m < 9; m++) {
                T t = 0.;
                t += p2[m] * T(H3); t += p1[m] * T(H3); t += cur[m] * T(H3);
                F[m * fs + c] = t;
            }
        }
#pragma unroll
        for (int m = 0; m < 9; m++) {
            p2[m] = p1[m];
            p1[m] = cur[m];
        }
    }
}

// A_ij = |S| S_ij and |S| of the interior from the velocities (pass 0 of
// k_dyn_mid: the same expressions).
template <typename T>
__global__ void k_dyn_strain(Grid g, Consts kc, const T *__restrict__ vel, T *__restrict__ A, T *__restrict__ Smag)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int i = blockIdx.z + 1;
    if (k > g.D || j > g.H) return;
    const long long fs = g.fstride, c = g.idx(i, j, k);
    if (!FSL_SPAN(c, -g.pi, g.pi, fs)) return;
    const long long dI = g.pi, dJ = g.pk;
    const T *uu = vel, *vv = vel + fs, *ww = vel + 2 * fs;
    const T du_dx = (uu[c + dI] - uu[c - dI]) * T(kc.r2dx);
    const T du_dy = (uu[c + dJ] - uu[c - dJ]) * T(kc.r2dy);
    const T du_dz = (uu[c + 1] - uu[c - 1]) * T(kc.r2dz);
    const T dv_dx = (vv[c + dI] - vv[c - dI]) * T(kc.r2dx);
    const T dv_dy = (vv[c + dJ] - vv[c - dJ]) * T(kc.r2dy);
    const T dv_dz = (vv[c + 1] - vv[c - 1]) * T(kc.r2dz);
    const T dw_dx = (ww[c + dI] - ww[c - dI]) * T(kc.r2dx);
    const T dw_dy = (ww[c + dJ] - ww[c - dJ]) * T(kc.r2dy);
    const T dw_dz = (ww[c + 1] - ww[c - 1]) * T(kc.r2dz);
    const T S11 = du_dx, S12 = T(0.5) * (du_dy + dv_dx), S13 = T(0.5) * (du_dz + dw_dx);
    const T S21 = S12, S22 = dv_dy, S23 = T(0.5) * (dv_dz + dw_dy);
    const T S31 = S13, S32 = S23, S33 = dw_dz;
    const T S = sqrt(2 * (S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 + S31 * S31 +
                          S32 * S32 + S33 * S33));
    A[c] = S * S11; A[fs + c] = S * S12; A[2 * fs + c] = S * S13;
    A[3 * fs + c] = S * S22; A[4 * fs + c] = S * S23; A[5 * fs + c] = S * S33;
    Smag[c] = S;
}

template <typename T, int TJ>
__global__ void __launch_bounds__(32 * TJ)
    k_dyn_filterA_final(Grid g, Consts kc, int seg, const double *__restrict__ rho, const T *__restrict__ F,
                        const T *__restrict__ A, const T *__restrict__ Smag, T *__restrict__ mu,
                        float *__restrict__ cd)
{
    __shared__ T qa[TJ + 2][34][6];
    __shared__ T t1[TJ][34][6];
    const int L = g.L, H = g.H, D = g.D;
    const int l = threadIdx.x, r = threadIdx.y, tid = r * 32 + l, nt = 32 * TJ;
    const int k0 = 1 + blockIdx.x * 32, j0 = 1 + blockIdx.y * TJ;
    const int j = j0 + r, k = k0 + l;
    const int i0 = 1 + blockIdx.z * seg, i1 = min(L, i0 + seg - 1);
    const long long fs = g.fstride;
    const bool own = j <= H && k <= D;
    T p2[6], p1[6], cur[6];
#pragma unroll
    for (int m = 0; m < 6; m++) p2[m] = p1[m] = cur[m] = T(0.);
    constexpr int NP = ((TJ + 2) * 34 + 32 * TJ - 1) / (32 * TJ);
    T pre[NP][6];
    auto issue = [&](int ip) {
#pragma unroll
        for (int s = 0; s < NP; s++) {
            const int e = tid + s * nt;
            const int rr = e / 34, cc = e % 34, jj = j0 - 1 + rr, kk = k0 - 1 + cc;
#pragma unroll
            for (int m = 0; m < 6; m++) pre[s][m] = T(0.);
            if (e < (TJ + 2) * 34 && ip >= 1 && ip <= L && jj <= H + 1 && kk <= D + 1) {
                const long long q = FSL_CELL(g.idx(ip, jj, kk), fs);
#pragma unroll
                for (int m = 0; m < 6; m++) pre[s][m] = A[m * fs + q];
            }
        }
    };
    issue(i0 - 1);
    for (int ip = i0 - 1; ip <= i1 + 1; ip++) {
        if (ip >= 1 && ip <= L) { // A is zero on the planes 0 and L+1
#pragma unroll
            for (int s = 0; s < NP; s++) {
                const int e = tid + s * nt;
                if (e < (TJ + 2) * 34) {
                    const int rr = e / 34, cc = e % 34;
#pragma unroll
                    for (int m = 0; m < 6; m++) qa[rr][cc][m] = pre[s][m];
                }
            }
            issue(ip + 1);
            __syncthreads();
            for (int e = tid; e < TJ * 34; e += nt) {
                const int rr = e / 34, cc = e % 34, jj = j0 + rr, kk = k0 - 1 + cc;
                const bool in = jj <= H && kk <= D;
#pragma unroll
                for (int m = 0; m < 6; m++) {
                    T t = 0.;
                    if (in) {
                        t += qa[rr][cc][m] * T(H3); t += qa[rr + 1][cc][m] * T(H3); t += qa[rr + 2][cc][m] * T(H3);
                    }
                    t1[rr][cc][m] = t;
                }
            }
            __syncthreads();
            if (own) {
#pragma unroll
                for (int m = 0; m < 6; m++) {
                    T t = 0.;
                    t += t1[r][l][m] * T(H3); t += t1[r][l + 1][m] * T(H3); t += t1[r][l + 2][m] * T(H3);
                    cur[m] = t;
                }
            }
            __syncthreads();
        } else {
#pragma unroll
            for (int m = 0; m < 6; m++) cur[m] = T(0.);
            if (ip == 0) issue(1); // the march starts on plane 0 (i0 = 1)
        }
        const int io = ip - 1;
        if (io >= i0 && io <= i1 && own) {
            T Ah[6];
#pragma unroll
            for (int m = 0; m < 6; m++) {
                T t = 0.;
                t += p2[m] * T(H3); t += p1[m] * T(H3); t += cur[m] * T(H3);
                Ah[m] = t;
            }
            const long long c = FSL_CELL(g.idx(io, j, k), fs);
            (void)FSL_SPAN(c, -g.pi, g.pi, fs); // its strain stencil (the block barriers forbid a skip)
            // Leonard stress (src/turbulence.c:250-270)
            const T f0 = F[c], f1 = F[fs + c], f2 = F[2 * fs + c];
            T L11 = F[3 * fs + c] - f0 * f0, L12 = F[4 * fs + c] - f0 * f1, L13 = F[5 * fs + c] - f0 * f2;
            T L22 = F[6 * fs + c] - f1 * f1, L23 = F[7 * fs + c] - f1 * f2, L33 = F[8 * fs + c] - f2 * f2;
            // |S^| S^ from the filtered velocities (pass 1 of k_dyn_mid)
            const long long dI = g.pi, dJ = g.pk;
            const T *uu = F, *vv = F + fs, *ww = F + 2 * fs;
            const T du_dx = (uu[c + dI] - uu[c - dI]) * T(kc.r2dx);
            const T du_dy = (uu[c + dJ] - uu[c - dJ]) * T(kc.r2dy);
            const T du_dz = (uu[c + 1] - uu[c - 1]) * T(kc.r2dz);
            const T dv_dx = (vv[c + dI] - vv[c - dI]) * T(kc.r2dx);
            const T dv_dy = (vv[c + dJ] - vv[c - dJ]) * T(kc.r2dy);
            const T dv_dz = (vv[c + 1] - vv[c - 1]) * T(kc.r2dz);
            const T dw_dx = (ww[c + dI] - ww[c - dI]) * T(kc.r2dx);
            const T dw_dy = (ww[c + dJ] - ww[c - dJ]) * T(kc.r2dy);
            const T dw_dz = (ww[c + 1] - ww[c - 1]) * T(kc.r2dz);
            const T S11 = du_dx, S12 = T(0.5) * (du_dy + dv_dx), S13 = T(0.5) * (du_dz + dw_dx);
            const T S21 = S12, S22 = dv_dy, S23 = T(0.5) * (dv_dz + dw_dy);
            const T S31 = S13, S32 = S23, S33 = dw_dz;
            const T Sh = sqrt(2 * (S11 * S11 + S12 * S12 + S13 * S13 + S21 * S21 + S22 * S22 + S23 * S23 +
                                   S31 * S31 + S32 * S32 + S33 * S33));
            // M_ij, coefficient, mu_SGS (src/turbulence.c:398-445; k_dyn_final)
            const T DD = T(kc.DD);
            const T M11 = DD * (4 * (Sh * S11) - Ah[0]);
            const T M12 = DD * (4 * (Sh * S12) - Ah[1]);
            const T M13 = DD * (4 * (Sh * S13) - Ah[2]);
            const T M22 = DD * (4 * (Sh * S22) - Ah[3]);
            const T M23 = DD * (4 * (Sh * S23) - Ah[4]);
            const T M33 = DD * (4 * (Sh * S33) - Ah[5]);
            const T tr = T(-(1.0 / 3.0)) * (L11 + L22 + L33);
            L11 += tr; L22 += tr; L33 += tr;
            const T LLMM = (L11 * M11 + L12 * M12 + L13 * M13 + L12 * M12 + L22 * M22 + L23 * M23 + L13 * M13 +
                            L23 * M23 + L33 * M33);
            const T MMMM = (M11 * M11 + M12 * M12 + M13 * M13 + M12 * M12 + M22 * M22 + M23 * M23 + M13 * M13 +
                            M23 * M23 + M33 * M33);
            T Cd = T(-0.5) * (LLMM / (MMMM + T(1e-30)));
            if (Cd > T(0.15)) Cd = T(0.15);
            else if (Cd < T(0.0)) Cd = T(0.0);
            mu[c] = T(rho[c]) * Cd * DD * Smag[c];
            if (cd) cd[c] = (float)Cd;
        }
#pragma unroll
        for (int m = 0; m < 6; m++) {
            p2[m] = p1[m];
            p1[m] = cur[m];
        }
    }
}

inline dim3 cells_grid3(dim3 b, int ni, int nj, int nk)
{
    return dim3((unsigned)((nk + b.x - 1) / b.x), (unsigned)((nj + b.y - 1) / b.y), (unsigned)ni);
}

// Scratch fields of one evaluation (each `fstride` elements of T).
template <typename T> struct Scratch {
    T *vel, *t1, *t2, *A, *Lst, *B, *S;
};

// The nine launches of one evaluation on `st`: velocities, the filter of the
// velocities and their products (y, z, x), Leonard stress, |S| S and |S^| S^,
// the filter of A (y, z, x) and the coefficient; mu in T, Cd as FP32 (or not).
template <typename T>
void sequence(const Grid &g, const Consts &k, const Scratch<T> &s, const double *U, T *mu, float *cd,
              cudaStream_t st)
{
    const long long ncell = (long long)(g.L + 2) * g.pi;
    k_dyn_vel<T><<<(unsigned)std::min<long long>((ncell + 255) / 256, 148LL * 16), 256, 0, st>>>(g, U, s.vel);
    const dim3 b(32, 4, 1);
    // velocity and product filters: y over i in [0,L] j in [1,H] k in [0,D]
    k_filt_y_vel<T><<<cells_grid3(b, g.L + 1, g.H, g.D + 1), b, 0, st>>>(g, s.vel, s.t1);
    k_filt_z<T><<<cells_grid3(b, g.L + 1, g.H + 1, g.D), b, 0, st>>>(g, 9, s.t1, s.t2);
    k_filt_x<T><<<cells_grid3(b, g.L, g.H + 1, g.D + 1), b, 0, st>>>(g, 9, s.t2, s.t1);
    k_dyn_mid<T><<<cells_grid3(b, g.L, g.H, g.D), b, 0, st>>>(g, k, s.vel, s.t1, s.Lst, s.A, s.B, s.S);
    // filter of A (pass-1 buffer reused; its zero bands are preserved)
    k_filt_y<T><<<cells_grid3(b, g.L + 1, g.H, g.D + 1), b, 0, st>>>(g, 6, s.A, s.t1);
    k_filt_z<T><<<cells_grid3(b, g.L + 1, g.H + 1, g.D), b, 0, st>>>(g, 6, s.t1, s.t2);
    k_filt_x<T><<<cells_grid3(b, g.L, g.H + 1, g.D + 1), b, 0, st>>>(g, 6, s.t2, s.t1);
    k_dyn_final<T><<<cells_grid3(b, g.L, g.H, g.D), b, 0, st>>>(g, k, U, s.Lst, s.B, s.t1, s.S, mu, cd);
}

// The fused evaluation: velocities, the nine-field filter, A and |S|, the
// filter of A with the coefficient and mu_SGS -- four launches.
template <typename T>
void sequence_fused(const Grid &g, const Consts &k, const Scratch3<T> &s, const double *U, T *mu, float *cd,
                    cudaStream_t st)
{
    constexpr int TJ = 8, SEG = 32;
    const long long ncell = (long long)(g.L + 2) * g.pi;
    k_dyn_vel<T><<<(unsigned)std::min<long long>((ncell + 255) / 256, 148LL * 16), 256, 0, st>>>(g, U, s.vel);
    const dim3 bt(32, TJ, 1);
    const dim3 g9((unsigned)((g.D + 1 + 31) / 32), (unsigned)((g.H + TJ - 1) / TJ), (unsigned)((g.L + 1 + SEG - 1) / SEG));
    k_dyn_filter9<T, TJ><<<g9, bt, 0, st>>>(g, SEG, s.vel, s.F);
    const dim3 b(32, 4, 1);
    k_dyn_strain<T><<<cells_grid3(b, g.L, g.H, g.D), b, 0, st>>>(g, k, s.vel, s.A, s.S);
    const dim3 g6((unsigned)((g.D + 31) / 32), (unsigned)((g.H + TJ - 1) / TJ), (unsigned)((g.L + SEG - 1) / SEG));
    k_dyn_filterA_final<T, TJ><<<g6, bt, 0, st>>>(g, k, SEG, U, s.F, s.A, s.S, mu, cd);
}

} // namespace dyn
} // namespace fsl
