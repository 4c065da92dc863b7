// flopcount.cu -- exact operation counts of one cell-stage of the explicit
// step, from the step's own arithmetic templates (fsl_phys.cuh) instantiated
// on the host with a counting number type.  Host code only.
//
// Two compositions of the same templates per interior cell and RK stage:
//  * "reference": as src/ evaluates it -- primitives and the three
//    characteristic sweeps once per cell (src/reconstruction.c:26-345); per
//    face (one x, y and z face per cell) the two adjacent cells' velocities by
//    division and the eight tangential neighbours' by reciprocal
//    (src/fluxes.c:117-142), the Riemann solve, gradients and flux assembly,
//    the face SGS viscosity average (:191); the stage combination
//    (src/evolution.c:29-161, averaged over the three stages).
//  * "fused": as the fused stage kernel evaluates it per output cell -- the
//    primitives twice (y/z sweeps of plane i, x sweep of plane i+1), the
//    three sweeps, one velocity set of each form and one face viscosity
//    average per cell (shared by the faces through on-chip memory), three
//    face fluxes, the same combination.  The plain FP64 kernel.
//  * "fused_fp32": the same with the FP32 bulk's regrouped sweeps and paired
//    limiter (recon_sweep_grouped, minmod2).
// Sign flips and absolute values are operand modifiers and are not counted;
// selects are not arithmetic.  Output: one JSON line.
#include <cmath>
#include <cstdio>

#include "fsl_phys.cuh"

namespace cnt {

struct Ops {
    long long add, mul, div, sqrt, cmp;
};
static Ops ops;

struct R {
    double v;
    constexpr R(double x = 0.0) : v(x) {}
};
inline R operator+(R a, R b) { ops.add++; return R(a.v + b.v); }
inline R operator-(R a, R b) { ops.add++; return R(a.v - b.v); }
inline R operator*(R a, R b) { ops.mul++; return R(a.v * b.v); }
inline R operator/(R a, R b) { ops.div++; return R(a.v / b.v); }
inline R operator-(R a) { return R(-a.v); }
inline R &operator+=(R &a, R b) { a = a + b; return a; }
inline R &operator-=(R &a, R b) { a = a - b; return a; }
inline bool operator>(R a, R b) { ops.cmp++; return a.v > b.v; }
inline bool operator<(R a, R b) { ops.cmp++; return a.v < b.v; }
inline bool operator>=(R a, R b) { ops.cmp++; return a.v >= b.v; }
inline bool operator<=(R a, R b) { ops.cmp++; return a.v <= b.v; }
inline R sqrt(R a) { ops.sqrt++; return R(std::sqrt(a.v)); }
inline R fabs(R a) { return R(std::fabs(a.v)); }
inline R fmin(R a, R b) { ops.cmp++; return R(std::fmin(a.v, b.v)); }
inline R copysign(R a, R b) { return R(std::copysign(a.v, b.v)); }

} // namespace cnt

using cnt::R;

struct KCst {
    double rdx = 1, rdy = 1, rdz = 1, r4dx = .25, r4dy = .25, r4dz = .25;
    double mu_L = 1e-3, lambda_L = 1.4, cp_Pr_T = 1250.;
};

static void state(R *u, double a)
{
    const double r = 1.0 + 0.1 * a, vx = 100. + 10. * a, vy = -5. + a, vz = 3. - a, p = 1e5 * (1. + 0.01 * a);
    u[0] = r; u[1] = r * vx; u[2] = r * vy; u[3] = r * vz; u[4] = p / 0.4 + 0.5 * r * (vx * vx + vy * vy + vz * vz);
}

static cnt::Ops take()
{
    cnt::Ops o = cnt::ops;
    cnt::ops = cnt::Ops{0, 0, 0, 0, 0};
    return o;
}

// primitives + the three sweeps of one cell
static void sweeps(int nconsts)
{
    fsl::CellC<R> c;
    state(c.u, 0.0);
    R fw[5], bw[5], hi[5], lo[5];
    state(fw, 0.3);
    state(bw, -0.2);
    for (int n = 0; n < nconsts; n++) fsl::cell_consts(c);
    fsl::recon_x(c, fw, bw, hi, lo);
    fsl::recon_y(c, fw, bw, hi, lo);
    fsl::recon_z(c, fw, bw, hi, lo);
}

// the same with the FP32 bulk's regrouped sweeps
static void sweeps_grouped(int nconsts)
{
    fsl::CellC<R> c;
    state(c.u, 0.0);
    R fw[5], bw[5], hi[5], lo[5];
    state(fw, 0.3);
    state(bw, -0.2);
    for (int n = 0; n < nconsts; n++) fsl::cell_consts(c);
    fsl::recon_sweep_grouped<R, 1, 2, 3>(c, c.U, c.V, c.W, c.bb, c.cc, c.dd, c.u_hh, c.v_hh, c.w_hh, c.u_ee,
                                         c.v_ee, c.w_ee, fw, bw, hi, lo);
    fsl::recon_sweep_grouped<R, 2, 3, 1>(c, c.V, c.W, c.U, c.cc, c.dd, c.bb, c.v_hh, c.w_hh, c.u_hh, c.v_ee,
                                         c.w_ee, c.u_ee, fw, bw, hi, lo);
    fsl::recon_sweep_grouped<R, 3, 1, 2>(c, c.W, c.U, c.V, c.dd, c.bb, c.cc, c.w_hh, c.u_hh, c.v_hh, c.w_ee,
                                         c.u_ee, c.w_ee, fw, bw, hi, lo);
}

// one face of normal N from precomputed velocities
template <int N> static void face()
{
    const KCst kc;
    R Lm[5], Rp[5], vm[4], vp[4], t[8][3], F[5];
    state(Lm, 0.1);
    state(Rp, -0.1);
    for (int q = 0; q < 4; q++) { vm[q] = R(1.0 + q); vp[q] = R(2.0 + q); }
    for (int a = 0; a < 8; a++)
        for (int q = 0; q < 3; q++) t[a][q] = R(0.5 * a + q);
    const R muT = R(1e-4);
    take();
    fsl::fused_face<R, N>(Lm, Rp, vm, vm[3], vp, vp[3], t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7], muT, kc, F);
}

static void velocities(int ndiv, int nrcp)
{
    R u[5], o[4], T;
    state(u, 0.05);
    for (int n = 0; n < ndiv; n++) fsl::vel_div(u[0], u[1], u[2], u[3], u[4], o, T);
    for (int n = 0; n < nrcp; n++) fsl::vel_rcp(u[0], u[1], u[2], u[3], o);
}

// the stage combination of src/evolution.c for one variable, stage s
static void combine(int s)
{
    const R dtx(1e-3), dty(1e-3), dtz(1e-3), b0(1.), un(1.), f[6] = {1, 2, 3, 4, 5, 6};
    const R X = dtx * (f[0] - f[1]), Y = dty * (f[2] - f[3]), Z = dtz * (f[4] - f[5]);
    if (s == 1) (void)(b0 + X + Y + Z);
    else if (s == 2) (void)(R(0.75) * un + R(0.25) * (b0 + X + Y + Z));
    else (void)(R(1. / 3.) * un + R(2. / 3.) * (b0 + X + Y + Z));
}

static void add(cnt::Ops &a, const cnt::Ops &b, double w = 1.0)
{
    a.add += (long long)(w * b.add); a.mul += (long long)(w * b.mul); a.div += (long long)(w * b.div);
    a.sqrt += (long long)(w * b.sqrt); a.cmp += (long long)(w * b.cmp);
}

static void print(const char *name, const cnt::Ops &o, bool comma)
{
    std::printf("\"%s\": {\"add\": %lld, \"mul\": %lld, \"div\": %lld, \"sqrt\": %lld, \"cmp\": %lld, "
                "\"flops\": %lld}%s",
                name, o.add, o.mul, o.div, o.sqrt, o.cmp, o.add + o.mul + o.div + o.sqrt, comma ? ", " : "");
}

int main()
{
    take();
    sweeps(1);
    const cnt::Ops sw1 = take();
    sweeps(2);
    const cnt::Ops sw2 = take();
    sweeps_grouped(2);
    const cnt::Ops sw32 = take();
    face<1>();
    const cnt::Ops fx = take();
    face<2>();
    const cnt::Ops fy = take();
    face<3>();
    const cnt::Ops fz = take();
    velocities(2, 8);
    const cnt::Ops vref = take();
    velocities(1, 1);
    const cnt::Ops vfus = take();
    cnt::Ops comb{0, 0, 0, 0, 0};
    for (int s = 1; s <= 3; s++) {
        for (int q = 0; q < 5; q++) combine(s);
        add(comb, take(), 1.0 / 3.0);
    }
    // face SGS viscosity average 0.5 (mu_a + mu_b): one add, one mul
    const cnt::Ops muavg{1, 1, 0, 0, 0};

    cnt::Ops ref{0, 0, 0, 0, 0}, fus{0, 0, 0, 0, 0}, f32{0, 0, 0, 0, 0};
    add(ref, sw1);
    add(ref, fx); add(ref, fy); add(ref, fz);
    add(ref, vref, 3.0);
    add(ref, muavg, 3.0);
    add(ref, comb);
    add(fus, sw2);
    add(fus, fx); add(fus, fy); add(fus, fz);
    add(fus, vfus);
    add(fus, muavg);
    add(fus, comb);
    add(f32, sw32);
    add(f32, fx); add(f32, fy); add(f32, fz);
    add(f32, vfus);
    add(f32, muavg);
    add(f32, comb);
    std::printf("{");
    print("reference", ref, true);
    print("fused", fus, true);
    print("fused_fp32", f32, true);
    print("sweeps", sw1, true);
    print("face_x", fx, true);
    print("face_y", fy, true);
    print("face_z", fz, true);
    print("combination", comb, false);
    std::printf("}\n");
    return 0;
}
