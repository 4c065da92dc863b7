// fsl_phys.cuh -- device arithmetic of the explicit step, templated on the
// compute type T (double for the plain method, float for the FP32 bulk).
//
// Every expression keeps the reference's evaluation order; translation units
// that instantiate T = double are compiled with --fmad=false so that the plain
// method rounds exactly like the reference's serial CPU code (IEEE division
// and square root are the CUDA defaults for double).
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

// Arithmetic templates callable from host code too (an instrumented
// instantiation counts their operations; the kernels use T = double, float).
#define FSL_HD __host__ __device__ __forceinline__

namespace fsl {

// gas and scheme constants, src/def.h:25-45
template <typename T> struct Kc {
    static constexpr T K = T(1.4);
    static constexpr T K_1 = T(0.4);
    static constexpr T NK_1 = T(-0.4);
    static constexpr T K05 = T(0.7);
    static constexpr T K_K_1 = T(3.5);
    static constexpr T K_1_2 = T(0.2);
    static constexpr T H_K_1 = T(1.25);
    static constexpr T R_VOZD = T(287.10);
    static constexpr T C1 = T(0.333333333333333);
    static constexpr T C2 = T(0.166666666666667);
    static constexpr T TWO_THIRDS = T(0.666666666666667);
};

// Chakravarthy-Osher minmod, compression 4 (src/reconstruction.c:17-24),
// written as selects: the same comparisons on the same values, so the same
// result, without data-dependent branches that split a warp.  (y = 0 never
// reaches |4y|: x y = 0 returns 0 first.)
template <typename T> FSL_HD T minmod(T x, T y)
{
    const T y4 = y * T(4.0);
    const T ay = (y4 > T(0)) ? y4 : -y4;
    const T r = (x > T(0)) ? ((x < ay) ? x : ay) : ((-x < ay) ? x : -ay);
    return (x * y <= T(0)) ? T(0) : r;
}

// minmod(a, b) and minmod(b, a) at once (the FP32 bulk): both are 0 when a b <= 0,
// else sign(a) min(|a|, 4|b|) and sign(b) min(|b|, 4|a|) -- exactly the
// values of the select form above (min, |.|, x4 and the sign copy are exact),
// with one product and one sign test for the pair.
template <typename T> FSL_HD void minmod2(T a, T b, T &ab, T &ba)
{
    const bool z = a * b <= T(0);
    const T fa = fabs(a), fb = fabs(b);
    const T m1 = copysign(fmin(fa, T(4) * fb), a);
    const T m2 = copysign(fmin(fb, T(4) * fa), b);
    ab = z ? T(0) : m1;
    ba = z ? T(0) : m2;
}

// Per-cell quantities shared by the three sweeps (src/reconstruction.c:63-88,
// :104, :142-145).
template <typename T> struct CellC {
    T u[5];
    T U, V, W, C;
    T aa, ll, ee, gg, hh, nn, S11;
    T bb, cc, dd;
    T u_hh, v_hh, w_hh, u_ee, v_ee, w_ee;
};

template <typename T> FSL_HD void cell_consts(CellC<T> &c)
{
    typedef Kc<T> k;
    T R = T(1.) / c.u[0];
    c.U = c.u[1] * R;
    c.V = c.u[2] * R;
    c.W = c.u[3] * R;
    T P = (c.u[4] - T(0.5) * (c.u[1] * c.u[1] + c.u[2] * c.u[2] + c.u[3] * c.u[3]) * R) * k::K_1;
    c.C = sqrt(k::K * P * R);
    T ff = c.U * c.U + c.V * c.V + c.W * c.W;
    c.aa = k::K_1_2 * ff;
    c.bb = k::NK_1 * c.U;
    c.cc = k::NK_1 * c.V;
    c.dd = k::NK_1 * c.W;
    c.ll = T(1.) / (c.C + c.C);
    c.ee = c.ll / c.C;
    c.gg = -ff * c.ee;
    c.hh = -(c.ee + c.ee);
    c.S11 = c.aa - c.C * c.C;
    c.u_hh = c.U * c.hh;
    c.v_hh = c.V * c.hh;
    c.w_hh = c.W * c.hh;
    c.u_ee = c.U * c.ee;
    c.v_ee = c.V * c.ee;
    c.w_ee = c.W * c.ee;
    c.nn = T(-0.5) * c.gg;
}

// The sweep below with its characteristic rows and face coefficients
// regrouped, for the FP32 bulk (which does not follow the reference's
// rounding): with d the forward (or backward) differences,
//   A = aa d1 + bn d2 + K_1 d5 + bt1 d3 + bt2 d4,  B = C (d2 - vn d1),
//   M1 = A - C^2 d1,  M4 = A + B,  M5 = A - B
// (S41 = aa - C vn, S42 = bn + C, S51 = aa + C vn, S52 = bn - C, S11 = aa - C^2),
// and on the faces n_ee (k4 + k5) + ll (k4 - k5) for _S24 k4 + _S25 k5 and
// (nn + H_K_1)(k4 + k5) + mm (k4 - k5) for _S54 k4 + _S55 k5.  The same
// scheme in fewer operations.
template <typename T, int N, int T1, int T2>
FSL_HD void recon_sweep_grouped(const CellC<T> &c, T vn, T vt1, T vt2, T bn, T bt1, T bt2, T n_hh, T t1_hh,
                                T t2_hh, T n_ee, T t1_ee, T t2_ee, const T *fw, const T *bw, T *hi, T *lo)
{
    typedef Kc<T> k;
    const T *u = c.u;
    const T C = c.C, C2 = c.aa - c.S11;
    T M[5], W[5];
    {
        const T d1 = fw[0] - u[0], d2 = fw[1] - u[N], d3 = fw[2] - u[T1], d4 = fw[3] - u[T2], d5 = fw[4] - u[4];
        const T A = c.aa * d1 + bn * d2 + k::K_1 * d5 + bt1 * d3 + bt2 * d4;
        const T B = C * (d2 - vn * d1);
        M[0] = A - C2 * d1; M[1] = d3 - vt1 * d1; M[2] = d4 - vt2 * d1; M[3] = A + B; M[4] = A - B;
    }
    {
        const T d1 = u[0] - bw[0], d2 = u[N] - bw[1], d3 = u[T1] - bw[2], d4 = u[T2] - bw[3], d5 = u[4] - bw[4];
        const T A = c.aa * d1 + bn * d2 + k::K_1 * d5 + bt1 * d3 + bt2 * d4;
        const T B = C * (d2 - vn * d1);
        W[0] = A - C2 * d1; W[1] = d3 - vt1 * d1; W[2] = d4 - vt2 * d1; W[3] = A + B; W[4] = A - B;
    }
    T Ml[5], Wl[5];
#pragma unroll
    for (int q = 0; q < 5; q++) minmod2(M[q], W[q], Ml[q], Wl[q]);
    const T mm = vn * c.ll, e45 = c.nn + k::H_K_1;
    {
        const T k1 = Ml[0] * k::C1 + Wl[0] * k::C2, k2 = Ml[1] * k::C1 + Wl[1] * k::C2;
        const T k3 = Ml[2] * k::C1 + Wl[2] * k::C2, k4 = Ml[3] * k::C1 + Wl[3] * k::C2;
        const T k5 = Ml[4] * k::C1 + Wl[4] * k::C2;
        const T ks = k4 + k5, kd = k4 - k5;
        hi[0] = u[0] + c.hh * k1 + c.ee * ks;
        hi[N] = u[N] + n_hh * k1 + n_ee * ks + c.ll * kd;
        hi[T1] = u[T1] + t1_hh * k1 + k2 + t1_ee * ks;
        hi[T2] = u[T2] + t2_hh * k1 + k3 + t2_ee * ks;
        hi[4] = u[4] + c.gg * k1 + vt1 * k2 + vt2 * k3 + e45 * ks + mm * kd;
    }
    {
        const T k1 = Ml[0] * k::C2 + Wl[0] * k::C1, k2 = Ml[1] * k::C2 + Wl[1] * k::C1;
        const T k3 = Ml[2] * k::C2 + Wl[2] * k::C1, k4 = Ml[3] * k::C2 + Wl[3] * k::C1;
        const T k5 = Ml[4] * k::C2 + Wl[4] * k::C1;
        const T ks = k4 + k5, kd = k4 - k5;
        lo[0] = u[0] - (c.hh * k1 + c.ee * ks);
        lo[N] = u[N] - (n_hh * k1 + n_ee * ks + c.ll * kd);
        lo[T1] = u[T1] - (t1_hh * k1 + k2 + t1_ee * ks);
        lo[T2] = u[T2] - (t2_hh * k1 + k3 + t2_ee * ks);
        lo[4] = u[4] - (c.gg * k1 + vt1 * k2 + vt2 * k3 + e45 * ks + mm * kd);
    }
}

// One sweep of the characteristic reconstruction.  N = index of the normal
// momentum in u[] (1..3); T1, T2 = tangential momenta in the reference's
// permuted order (x: 2 3 4 -> 1 2 3; y: 3 4 2 -> 2 3 1; z: 4 2 3 -> 3 1 2).
// fw/bw: forward/backward neighbour values in the order (rho, N, T1, T2, E).
// hi: state on the face towards the forward neighbour, lo: towards the
// backward neighbour, natural variable order.  t2_ee is the coefficient the
// reference applies to the T2 momentum (the z sweep uses w_ee for rho v,
// src/reconstruction.c:328,340).
template <typename T, int N, int T1, int T2>
FSL_HD void recon_sweep(const CellC<T> &c, T vn, T vt1, T vt2, T bn, T bt1, T bt2,
                                            T n_hh, T t1_hh, T t2_hh, T n_ee, T t1_ee, T t2_ee,
                                            const T *fw, const T *bw, T *hi, T *lo)
{
    if constexpr (std::is_same<T, float>::value) {
        recon_sweep_grouped<T, N, T1, T2>(c, vn, vt1, vt2, bn, bt1, bt2, n_hh, t1_hh, t2_hh, n_ee, t1_ee, t2_ee,
                                          fw, bw, hi, lo);
        return;
    }
    typedef Kc<T> k;
    const T *u = c.u;
    const T C = c.C;
    T m1, m2, m3, m4, m5, w1, w2, w3, w4, w5;
    T M1, M2, M3, M4, M5, W1, W2, W3, W4, W5;
    T _M1, _M2, _M3, _M4, _M5, _W1, _W2, _W3, _W4, _W5;
    T S12, S41, S42, S51, S52, _S24, _S25, _S54, _S55;
    T k1, k2, k3, k4, k5, kk, mm;
    mm = vn * c.ll;
    m1 = fw[0] - u[0]; m2 = fw[1] - u[N]; m3 = fw[2] - u[T1]; m4 = fw[3] - u[T2]; m5 = fw[4] - u[4];
    w1 = u[0] - bw[0]; w2 = u[N] - bw[1]; w3 = u[T1] - bw[2]; w4 = u[T2] - bw[3]; w5 = u[4] - bw[4];
    S41 = c.aa - (kk = C * vn);
    S51 = c.aa + kk;
    S12 = S42 = S52 = bn;
    S42 += C;
    S52 -= C;
    kk = k::K_1 * m5; k2 = bt1 * m3; k3 = bt2 * m4;
    M1 = c.S11 * m1 + S12 * m2 + k2 + k3 + kk;
    M2 = -vt1 * m1 + m3;
    M3 = -vt2 * m1 + m4;
    M4 = S41 * m1 + S42 * m2 + k2 + k3 + kk;
    M5 = S51 * m1 + S52 * m2 + k2 + k3 + kk;
    kk = k::K_1 * w5; k2 = bt1 * w3; k3 = bt2 * w4;
    W1 = c.S11 * w1 + S12 * w2 + k2 + k3 + kk;
    W2 = -vt1 * w1 + w3;
    W3 = -vt2 * w1 + w4;
    W4 = S41 * w1 + S42 * w2 + k2 + k3 + kk;
    W5 = S51 * w1 + S52 * w2 + k2 + k3 + kk;
    _M1 = minmod(M1, W1); _M2 = minmod(M2, W2); _M3 = minmod(M3, W3);
    _M4 = minmod(M4, W4); _M5 = minmod(M5, W5);
    _W1 = minmod(W1, M1); _W2 = minmod(W2, M2); _W3 = minmod(W3, M3);
    _W4 = minmod(W4, M4); _W5 = minmod(W5, M5);
    _S24 = n_ee + c.ll; _S25 = n_ee - c.ll;
    _S54 = _S55 = c.nn + k::H_K_1;
    _S54 += mm; _S55 -= mm;
    k1 = _M1 * k::C1 + _W1 * k::C2; k2 = _M2 * k::C1 + _W2 * k::C2; k3 = _M3 * k::C1 + _W3 * k::C2;
    k4 = _M4 * k::C1 + _W4 * k::C2; k5 = _M5 * k::C1 + _W5 * k::C2;
    kk = k4 + k5;
    hi[0] = u[0] + c.hh * k1 + c.ee * kk;
    hi[N] = u[N] + n_hh * k1 + _S24 * k4 + _S25 * k5;
    hi[T1] = u[T1] + t1_hh * k1 + k2 + t1_ee * kk;
    hi[T2] = u[T2] + t2_hh * k1 + k3 + t2_ee * kk;
    hi[4] = u[4] + c.gg * k1 + vt1 * k2 + vt2 * k3 + _S54 * k4 + _S55 * k5;
    k1 = _M1 * k::C2 + _W1 * k::C1; k2 = _M2 * k::C2 + _W2 * k::C1; k3 = _M3 * k::C2 + _W3 * k::C1;
    k4 = _M4 * k::C2 + _W4 * k::C1; k5 = _M5 * k::C2 + _W5 * k::C1;
    kk = k4 + k5;
    lo[0] = u[0] - c.hh * k1 - c.ee * kk;
    lo[N] = u[N] - n_hh * k1 - _S24 * k4 - _S25 * k5;
    lo[T1] = u[T1] - t1_hh * k1 - k2 - t1_ee * kk;
    lo[T2] = u[T2] - t2_hh * k1 - k3 - t2_ee * kk;
    lo[4] = u[4] - c.gg * k1 - vt1 * k2 - vt2 * k3 - _S54 * k4 - _S55 * k5;
}

// x, y and z sweeps with the reference's permutations.
template <typename T> FSL_HD void recon_x(const CellC<T> &c, const T *fw, const T *bw, T *hi, T *lo)
{
    recon_sweep<T, 1, 2, 3>(c, c.U, c.V, c.W, c.bb, c.cc, c.dd, c.u_hh, c.v_hh, c.w_hh, c.u_ee, c.v_ee,
                            c.w_ee, fw, bw, hi, lo);
}
template <typename T> FSL_HD void recon_y(const CellC<T> &c, const T *fw, const T *bw, T *hi, T *lo)
{
    recon_sweep<T, 2, 3, 1>(c, c.V, c.W, c.U, c.cc, c.dd, c.bb, c.v_hh, c.w_hh, c.u_hh, c.v_ee, c.w_ee,
                            c.u_ee, fw, bw, hi, lo);
}
template <typename T> FSL_HD void recon_z(const CellC<T> &c, const T *fw, const T *bw, T *hi, T *lo)
{
    recon_sweep<T, 3, 1, 2>(c, c.W, c.U, c.V, c.dd, c.bb, c.cc, c.w_hh, c.u_hh, c.v_hh, c.w_ee, c.u_ee,
                            c.w_ee, fw, bw, hi, lo);
}

// PPM (project extension; the reference has only the scheme above): Colella
// & Woodward (1984) on the same characteristic variables, with cell i's
// transform (src/reconstruction.c:104-129) and inverse (:148-158).  Per
// characteristic field: monotonised-central slopes (CW84 eq. 1.8) of cells
// i-1, i, i+1, edge values a_{i+1/2} - a_i = 1/2 d_{i+1/2} - (da_{i+1} -
// da_i)/6 and a_{i-1/2} - a_i = -1/2 d_{i-1/2} - (da_i - da_{i-1})/6 (eq.
// 1.6), the monotonicity limiter (eq. 1.10); the same arithmetic as the
// oracle's restatement.
template <typename T> FSL_HD T ppm_mc(T a, T b)
{
    if constexpr (std::is_same<T, float>::value) {
        // FP32 bulk: the same value as a min and a sign copy
        const T m = fmin(fmin(T(0.5) * fabs(a + b), T(2.0) * fabs(a)), T(2.0) * fabs(b));
        return (a * b <= T(0.0)) ? T(0.0) : copysign(m, a);
    }
    T m = T(0.5) * fabs(a + b);
    const T ta = T(2.0) * fabs(a), tb = T(2.0) * fabs(b);
    m = (ta < m) ? ta : m;
    m = (tb < m) ? tb : m;
    return (a * b <= T(0.0)) ? T(0.0) : ((a > T(0.0)) ? m : -m);
}

template <typename T>
FSL_HD void char_fwd(const CellC<T> &c, T vn, T vt1, T vt2, T bn, T bt1, T bt2, const T *d, T *M)
{
    typedef Kc<T> k;
    if constexpr (std::is_same<T, float>::value) {
        // FP32 bulk: the rows regrouped as in recon_sweep_grouped
        const T A = c.aa * d[0] + bn * d[1] + k::K_1 * d[4] + bt1 * d[2] + bt2 * d[3];
        const T B = c.C * (d[1] - vn * d[0]);
        M[0] = A - (c.aa - c.S11) * d[0];
        M[1] = d[2] - vt1 * d[0];
        M[2] = d[3] - vt2 * d[0];
        M[3] = A + B;
        M[4] = A - B;
        return;
    }
    const T C = c.C;
    T S12, S41, S42, S51, S52, kk, k2, k3;
    S41 = c.aa - (kk = C * vn);
    S51 = c.aa + kk;
    S12 = S42 = S52 = bn;
    S42 += C;
    S52 -= C;
    kk = k::K_1 * d[4]; k2 = bt1 * d[2]; k3 = bt2 * d[3];
    M[0] = c.S11 * d[0] + S12 * d[1] + k2 + k3 + kk;
    M[1] = -vt1 * d[0] + d[2];
    M[2] = -vt2 * d[0] + d[3];
    M[3] = S41 * d[0] + S42 * d[1] + k2 + k3 + kk;
    M[4] = S51 * d[0] + S52 * d[1] + k2 + k3 + kk;
}

template <typename T, int N, int T1, int T2>
FSL_HD void char_inv(const CellC<T> &c, T vn, T vt1, T vt2, T n_hh, T t1_hh, T t2_hh, T n_ee,
                                         T t1_ee, T t2_ee, const T *q, T *out)
{
    typedef Kc<T> k;
    const T *u = c.u;
    if constexpr (std::is_same<T, float>::value) {
        // FP32 bulk: the face coefficients as sums and differences
        const T ks = q[3] + q[4], kd = q[3] - q[4];
        out[0] = u[0] + c.hh * q[0] + c.ee * ks;
        out[N] = u[N] + n_hh * q[0] + n_ee * ks + c.ll * kd;
        out[T1] = u[T1] + t1_hh * q[0] + q[1] + t1_ee * ks;
        out[T2] = u[T2] + t2_hh * q[0] + q[2] + t2_ee * ks;
        out[4] = u[4] + c.gg * q[0] + vt1 * q[1] + vt2 * q[2] + (c.nn + k::H_K_1) * ks + (vn * c.ll) * kd;
        return;
    }
    const T mm = vn * c.ll;
    T _S24, _S25, _S54, _S55, kk;
    _S24 = n_ee + c.ll; _S25 = n_ee - c.ll;
    _S54 = _S55 = c.nn + k::H_K_1;
    _S54 += mm; _S55 -= mm;
    kk = q[3] + q[4];
    out[0] = u[0] + c.hh * q[0] + c.ee * kk;
    out[N] = u[N] + n_hh * q[0] + _S24 * q[3] + _S25 * q[4];
    out[T1] = u[T1] + t1_hh * q[0] + q[1] + t1_ee * kk;
    out[T2] = u[T2] + t2_hh * q[0] + q[2] + t2_ee * kk;
    out[4] = u[4] + c.gg * q[0] + vt1 * q[1] + vt2 * q[2] + _S54 * q[3] + _S55 * q[4];
}

// m2, m1, p1, p2: the neighbours at -2, -1, +1, +2 in the sweep's order
// (rho, normal, t1, t2, E); hi, lo as recon_sweep.
template <typename T, int N, int T1, int T2>
FSL_HD void ppm_sweep(const CellC<T> &c, T vn, T vt1, T vt2, T bn, T bt1, T bt2, T n_hh,
                                          T t1_hh, T t2_hh, T n_ee, T t1_ee, T t2_ee, const T *m2, const T *m1,
                                          const T *p1, const T *p2, T *hi, T *lo)
{
    const T *u = c.u;
    const T uc[5] = {u[0], u[N], u[T1], u[T2], u[4]};
    T d[5], W0[5], W1[5], W2[5], W3[5], qR[5], qL[5];
#pragma unroll
    for (int v = 0; v < 5; v++) d[v] = m1[v] - m2[v];
    char_fwd(c, vn, vt1, vt2, bn, bt1, bt2, d, W0);
#pragma unroll
    for (int v = 0; v < 5; v++) d[v] = uc[v] - m1[v];
    char_fwd(c, vn, vt1, vt2, bn, bt1, bt2, d, W1);
#pragma unroll
    for (int v = 0; v < 5; v++) d[v] = p1[v] - uc[v];
    char_fwd(c, vn, vt1, vt2, bn, bt1, bt2, d, W2);
#pragma unroll
    for (int v = 0; v < 5; v++) d[v] = p2[v] - p1[v];
    char_fwd(c, vn, vt1, vt2, bn, bt1, bt2, d, W3);
#pragma unroll
    for (int v = 0; v < 5; v++) {
        const T dm = ppm_mc(W0[v], W1[v]), d0 = ppm_mc(W1[v], W2[v]), dp = ppm_mc(W2[v], W3[v]);
        T r = T(0.5) * W2[v] - (dp - d0) / T(6.0), l = T(-0.5) * W1[v] - (d0 - dm) / T(6.0);
        if constexpr (std::is_same<T, float>::value) {
            // FP32 bulk: |r| > 2|l| and |l| > 2|r| exclude each other unless
            // both are zero, which the flat case covers
            const bool flat = r * l >= T(0.0);
            const T ar = fabs(r), al = fabs(l);
            qR[v] = flat ? T(0.0) : (ar > T(2.0) * al ? T(-2.0) * l : r);
            qL[v] = flat ? T(0.0) : (al > T(2.0) * ar ? T(-2.0) * r : l);
            continue;
        }
        const bool flat = r * l >= T(0.0);
        const bool capR = !flat && fabs(r) > T(2.0) * fabs(l);
        const bool capL = !flat && !capR && fabs(l) > T(2.0) * fabs(r);
        const T r2 = flat ? T(0.0) : (capR ? T(-2.0) * l : r);
        const T l2 = flat ? T(0.0) : (capL ? T(-2.0) * r : l);
        qR[v] = r2;
        qL[v] = l2;
    }
    char_inv<T, N, T1, T2>(c, vn, vt1, vt2, n_hh, t1_hh, t2_hh, n_ee, t1_ee, t2_ee, qR, hi);
    char_inv<T, N, T1, T2>(c, vn, vt1, vt2, n_hh, t1_hh, t2_hh, n_ee, t1_ee, t2_ee, qL, lo);
}

template <typename T>
FSL_HD void ppm_x(const CellC<T> &c, const T *m2, const T *m1, const T *p1, const T *p2, T *hi, T *lo)
{
    ppm_sweep<T, 1, 2, 3>(c, c.U, c.V, c.W, c.bb, c.cc, c.dd, c.u_hh, c.v_hh, c.w_hh, c.u_ee, c.v_ee, c.w_ee, m2, m1,
                          p1, p2, hi, lo);
}
template <typename T>
FSL_HD void ppm_y(const CellC<T> &c, const T *m2, const T *m1, const T *p1, const T *p2, T *hi, T *lo)
{
    ppm_sweep<T, 2, 3, 1>(c, c.V, c.W, c.U, c.cc, c.dd, c.bb, c.v_hh, c.w_hh, c.u_hh, c.v_ee, c.w_ee, c.u_ee, m2, m1,
                          p1, p2, hi, lo);
}
template <typename T>
FSL_HD void ppm_z(const CellC<T> &c, const T *m2, const T *m1, const T *p1, const T *p2, T *hi, T *lo)
{
    ppm_sweep<T, 3, 1, 2>(c, c.W, c.U, c.V, c.dd, c.bb, c.cc, c.w_hh, c.u_hh, c.v_hh, c.w_ee, c.u_ee, c.w_ee, m2, m1,
                          p1, p2, hi, lo);
}

// Linearised characteristic Riemann solve on one face (src/fluxes.c:61-113,
// :230-282, :401-453).  N = normal direction 1..3.  Lm/Rp: minus/plus
// conserved states.  Returns interface density, pressure and velocity (the
// normal component from the solve, the tangential ones upwinded by its sign).
template <typename T, int N>
FSL_HD void riemann(const T *Lm, const T *Rp, T &Rho, T &Pr, T *vel)
{
    typedef Kc<T> k;
    T _R, _P, _C, _jo, _jp, _jm, RU, R_, P_, C_, jo_, jp_, jm_;
    T lv[3], rv[3];
    T Un, C, C_p, C_m, C_o, al_p, al_m, al_o, J_p, J_m, J_o, P;
    _R = Lm[0];
    lv[0] = Lm[1] / _R; lv[1] = Lm[2] / _R; lv[2] = Lm[3] / _R;
    _P = (Lm[4] - T(0.5) * _R * (lv[0] * lv[0] + lv[1] * lv[1] + lv[2] * lv[2])) * k::K_1;
    _C = sqrt(k::K * _P / _R);
    _jo = k::NK_1 * _P;
    _jp = lv[N - 1] + (RU = _P / (_R * _C));
    _jm = lv[N - 1] - RU;
    R_ = Rp[0];
    rv[0] = Rp[1] / R_; rv[1] = Rp[2] / R_; rv[2] = Rp[3] / R_;
    P_ = (Rp[4] - T(0.5) * R_ * (rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2])) * k::K_1;
    C_ = sqrt(k::K * P_ / R_);
    jo_ = k::NK_1 * P_;
    jp_ = rv[N - 1] + (RU = P_ / (R_ * C_));
    jm_ = rv[N - 1] - RU;
    Un = T(0.5) * (lv[N - 1] + rv[N - 1]);
    C = T(0.5) * (_C + C_);
    C_p = Un + C; C_m = Un - C; C_o = Un;
    // upwind choices of src/fluxes.c:90-108 as operand selects (one division
    // each on the chosen operands: the same arithmetic as the branches)
    const bool pp = C_p > T(0.), pm = C_m > T(0.), po = C_o > T(0.);
    al_p = k::K_1_2 * (pp ? (_jm - _jp) : (jm_ - jp_)) / (pp ? _jo : jo_);
    J_p = pp ? _jp : jp_;
    al_m = k::K_1_2 * (pm ? (_jp - _jm) : (jp_ - jm_)) / (pm ? _jo : jo_);
    J_m = pm ? _jm : jm_;
    al_o = k::K05 * (po ? (_jp - _jm) : (jp_ - jm_));
    al_o = -al_o * al_o;
    J_o = po ? _jo : jo_;
    P = (J_p - J_m) / (al_p - al_m);
    Un = J_p - al_p * P;
    Rho = (J_o - P) / al_o;
    Pr = P;
    const bool up = Un > T(0);
    vel[0] = up ? lv[0] : rv[0];
    vel[1] = up ? lv[1] : rv[1];
    vel[2] = up ? lv[2] : rv[2];
    vel[N - 1] = Un;
}

// Velocities by reciprocal, RU = 1./rho (src/fluxes.c:124-142).
template <typename T> FSL_HD void vel_rcp(T r, T mu_, T mv, T mw, T *o)
{
    T RU = T(1.) / r;
    o[0] = mu_ * RU; o[1] = mv * RU; o[2] = mw * RU;
}

// Velocities and temperature by division (src/fluxes.c:117-122).
template <typename T> FSL_HD void vel_div(T R_, T mu_, T mv, T mw, T E, T *o, T &Tt)
{
    typedef Kc<T> k;
    T U_ = mu_ / R_, V_ = mv / R_, W_ = mw / R_;
    T P_ = (E - T(0.5) * R_ * (U_ * U_ + V_ * V_ + W_ * W_)) * k::K_1;
    Tt = P_ / (k::R_VOZD * R_);
    o[0] = U_; o[1] = V_; o[2] = W_;
}

// Flux assembly of one face from the Riemann state, the face velocity
// gradient and the cell-centre velocities of the two adjacent cells
// (src/fluxes.c:185-220, :353-391, :524-568).  N = normal direction.
// g[a][b] = d u_a / d x_b.  fw/bw: velocities of the plus/minus cell.
template <typename T, int N>
FSL_HD void face_flux(T Rho, T P, const T *vel, const T (*g)[3], const T *fw, const T *bw,
                                          T Tp, T Tm, T mu_L, T mu_T, T lambda_L, T cp_Pr_T, T rdn, T *F)
{
    typedef Kc<T> k;
    T uu = T(0.5) * (fw[0] + bw[0]), vv = T(0.5) * (fw[1] + bw[1]), ww = T(0.5) * (fw[2] + bw[2]);
    T mu_E = mu_L + mu_T;
    T s0, s1, s2; // sigma_N{x,y,z}
    if (N == 1) {
        s0 = k::TWO_THIRDS * mu_E * (g[0][0] + g[0][0] - g[1][1] - g[2][2]);
        s1 = mu_E * (g[0][1] + g[1][0]);
        s2 = mu_E * (g[0][2] + g[2][0]);
    } else if (N == 2) {
        s0 = mu_E * (g[1][0] + g[0][1]);
        s1 = k::TWO_THIRDS * mu_E * (g[1][1] + g[1][1] - g[0][0] - g[2][2]);
        s2 = mu_E * (g[1][2] + g[2][1]);
    } else {
        s0 = mu_E * (g[2][0] + g[0][2]);
        s1 = mu_E * (g[2][1] + g[1][2]);
        s2 = k::TWO_THIRDS * mu_E * (g[2][2] + g[2][2] - g[0][0] - g[1][1]);
    }
    T lambda_E = lambda_L + mu_T * cp_Pr_T;
    T q = -lambda_E * (Tp - Tm) * rdn;
    T RU = Rho * vel[N - 1];
    F[0] = RU;
    F[1] = RU * vel[0] - s0;
    F[2] = RU * vel[1] - s1;
    F[3] = RU * vel[2] - s2;
    if (N == 1) F[1] = RU * vel[0] + P - s0;
    if (N == 2) F[2] = RU * vel[1] + P - s1;
    if (N == 3) F[3] = RU * vel[2] + P - s2;
    F[4] = vel[N - 1] * (k::K_K_1 * P + T(0.5) * Rho * (vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2])) -
           uu * s0 - vv * s1 - ww * s2 + q;
}

// The static Smagorinsky viscosity of one face (the reference's
// DynamicSmagorinskySGS 0 branch, src/fluxes.c:193-205 x, :362-374 y,
// :533-545 z; live in src-par/def.h:47): the mean density of the two cells
// beside the face times CsDD = Cs (dx dy dz)^(2/3) times |S| from the face
// velocity gradients g[a][b] = d u_a / d x_b, in the reference's order.
template <typename T> FSL_HD T static_mu_t(const T (*g)[3], T rr, T CsDD)
{
    const T S12 = T(0.5) * (g[0][1] + g[1][0]);
    const T S13 = T(0.5) * (g[0][2] + g[2][0]);
    const T S23 = T(0.5) * (g[1][2] + g[2][1]);
    const T S = sqrt(T(2) * (g[0][0] * g[0][0] + g[1][1] * g[1][1] + g[2][2] * g[2][2] +
                             T(2) * (S12 * S12 + S13 * S13 + S23 * S23)));
    return rr * CsDD * S;
}

// Flux of one face (src/fluxes.c): Riemann state from the two face states,
// viscous and heat flux from the two adjacent cells (vm/Tm minus side, vp/Tp
// plus side, by division) and the eight tangential neighbours (by
// reciprocal; P/M = plus/minus cell, h/l = +/- along the first (1) and
// second (2) tangential axis).  kc: grid spacings and transport constants
// (rdx.., r4dx.., mu_L, lambda_L, cp_Pr_T, CsDD).  muT is the face's SGS
// viscosity; with SST (static Smagorinsky) it is the mean density of the two
// cells beside the face, and the viscosity is formed here from the gradients.
template <typename T, int N, bool SST = false, typename KC>
FSL_HD void fused_face(const T *Lm, const T *Rp, const T *vm, T Tm, const T *vp, T Tp, const T *Ph1, const T *Mh1,
                       const T *Pl1, const T *Ml1, const T *Ph2, const T *Mh2, const T *Pl2, const T *Ml2, T muT,
                       const KC &kc, T *F)
{
    T Rho, P, vel[3];
    riemann<T, N>(Lm, Rp, Rho, P, vel);
    const int n0 = N - 1;
    const int t1 = (N == 1) ? 1 : 0;
    const int t2 = (N == 3) ? 1 : 2;
    const T rdn = T(N == 1 ? kc.rdx : N == 2 ? kc.rdy : kc.rdz);
    const T rt1 = T(N == 1 ? kc.r4dy : kc.r4dx);
    const T rt2 = T(N == 3 ? kc.r4dy : kc.r4dz);
    T gr[3][3];
#pragma unroll
    for (int q = 0; q < 3; q++) {
        gr[q][n0] = (vp[q] - vm[q]) * rdn;
        gr[q][t1] = (Ph1[q] + Mh1[q] - Pl1[q] - Ml1[q]) * rt1;
        gr[q][t2] = (Ph2[q] + Mh2[q] - Pl2[q] - Ml2[q]) * rt2;
    }
    if constexpr (SST) muT = static_mu_t<T>(gr, muT, T(kc.CsDD));
    face_flux<T, N>(Rho, P, vel, gr, vp, vm, Tp, Tm, T(kc.mu_L), muT, T(kc.lambda_L), T(kc.cp_Pr_T), rdn, F);
}

template <typename T> FSL_HD void vdiv(const T *U, T *o)
{
    T Tt;
    vel_div(U[0], U[1], U[2], U[3], U[4], o, Tt);
    o[3] = Tt;
}

// Courant number of one cell from its conserved variables: the reference's
// streamwise u dt/dx (src/helpers.c:31-43) or the acoustic sum
// dt((|u|+c)/dx + (|v|+c)/dy + (|w|+c)/dz) (a project extension, formed with
// the reciprocal ir = 1/rho: one division instead of four).  Every operation
// is an explicitly rounded FP64 intrinsic, so the value does not depend on
// the contraction flags of the translation unit: the standalone reduction and
// the fused stage kernels (FP64 and FP32 bulk) produce the same bits.
__device__ __forceinline__ double cell_courant_ir(int mode, double R, double ir, double mu, double mv, double mw,
                                                  double E, double dtx, double dty, double dtz)
{
    if (mode != 1) return __dmul_rn(__ddiv_rn(mu, R), dtx);
    const double Uv = __dmul_rn(mu, ir), V = __dmul_rn(mv, ir), W = __dmul_rn(mw, ir);
    const double q = __dadd_rn(__dadd_rn(__dmul_rn(Uv, Uv), __dmul_rn(V, V)), __dmul_rn(W, W));
    const double P = __dmul_rn(__dsub_rn(E, __dmul_rn(__dmul_rn(0.5, R), q)), 0.4);
    const double Cs = __dsqrt_rn(__dmul_rn(__dmul_rn(1.4, P), ir));
    return __dadd_rn(__dadd_rn(__dmul_rn(__dadd_rn(fabs(Uv), Cs), dtx), __dmul_rn(__dadd_rn(fabs(V), Cs), dty)),
                     __dmul_rn(__dadd_rn(fabs(W), Cs), dtz));
}
__device__ __forceinline__ double cell_courant(int mode, double R, double mu, double mv, double mw, double E,
                                               double dtx, double dty, double dtz)
{
    return cell_courant_ir(mode, R, mode == 1 ? __ddiv_rn(1.0, R) : 0.0, mu, mv, mw, E, dtx, dty, dtz);
}

} // namespace fsl
