// fsl_stage_wide.cuh -- the FP32-bulk fused RK3 stage kernel with a full-lane
// tile, for the reference reconstruction (src/reconstruction.c:26-345).
//
// The ring-tile kernel (fsl_stage.cuh) gives each of its 32 x TJE threads a
// cell of a tile that includes its own one-cell halo ring: the ring threads
// load and reconstruct, then idle through the x sweep, the three face fluxes
// and the stage combination, and a 30-wide tile leaves lanes empty where the
// domain's DEP is a multiple of 32.  Here every thread owns an interior
// column: a block of 16 warps x 32 lanes owns a 16 (y) x 32 (z) tile and the
// halo ring's work is handed out as whole-warp tasks:
//   - loads of the state halo (two rows and two columns on each side) and the
//     velocities of the one-cell ring: threads 0..195, one cell each;
//   - the y sweeps of the two halo rows and the z sweeps of the two halo
//     columns (warps 13, 14, 15; one warp-wide pass for both columns), one
//     plane ahead, after the stage combination of the plane before, so that
//     the sweep phase before a plane's first barrier has the own sweeps only;
//   - the fluxes of the tile's bottom y faces and left z faces (warps 12
//     and 11), between the two barriers.
// The tile's own faces (the y face above each cell, the z face beyond it,
// the x face ahead of it) are computed once each, as in the ring-tile kernel;
// the z faces exchange states and fluxes between neighbouring lanes by warp
// shuffles.  Arithmetic, boundary rules and the march along x (planes i+2 in
// flight while plane i is computed, two barriers per plane) are those of the
// ring-tile kernel.
//
// The grid is persistent: one block per SM (or fewer for small domains) takes
// its share of the domain's (tile, plane) pairs, so there is no tail wave.
// The pairs are ordered heads first: the first Hd planes of every tile, tile
// after tile, then the remaining planes of every tile.  With more blocks
// than tiles, block b < tiles takes the head of tile b and the other blocks
// share the tails (weighted: a tail block starts several segments); the head
// blocks start on neighbouring tiles at the same plane and march in step, so
// the halo planes one block reads were read by its neighbours moments before
// and come from L2 (tile-major ranges, out of step, measured 2.5 % slower).
#pragma once

#include "fsl_stage.cuh"

namespace fsl {
namespace wide {

using stage::Args;
using stage::BF;
using stage::load5;
using stage::recon_at;

constexpr int WJ = 16;  // tile rows (warps)
constexpr int WK = 32;  // tile columns (lanes)
constexpr int NT = WJ * WK;
constexpr int NHALO = 196; // state halo cells loaded per plane (see halo_cell)

template <typename T> struct Smem {
    T U[2][WJ + 4][WK + 4][5];  // state of planes i, i+1: rows -2..17, cols -2..33
    T R[3][WJ + 2][WK + 2][3];  // velocities by reciprocal, planes i-1, i, i+1: rows -1..16, cols -1..32
    T Dv[2][WJ + 2][WK + 2][5]; // velocities by division, T, face-averaged mu: planes i, i+1
    T Lo[WJ][WK][5];            // y sweep, state on the face below: rows 0..15
    T Fy[WJ + 1][WK][5];        // y flux of the face below row r (r = 0..16: faces j0-1/2 .. j0+15+1/2)
    // the halo sweeps, by plane parity (computed one plane ahead):
    T HyB[2][WK][5];            // y sweep of halo row -1, state on the face above it
    T LoH[2][WK][5];            // y sweep of halo row 16, state on the face below it
    T HzL[2][WJ][5];            // z sweep of halo column -1, state on the face beyond it
    T LzR[2][WJ][5];            // z sweep of halo column 32, state on the face before it
    T Lz0[WJ][5];               // z sweep of column 0, state on the face before it
    T FzL[WJ][5];               // z flux of the face before column 0
    double comax[WJ][WK];       // Courant maxima of the cells written
};

// Ring coordinates of state-halo cell h (0..195) of a tile: rows -2, -1, 16,
// 17 over the 32 columns (h < 128), columns -2, -1, 32, 33 over the 16 rows
// (h < 192), and the four corners of the one-cell ring (h < 196).  The
// velocity ring's halo (rows -1 and 16 over columns -1..32, columns -1 and
// 32 over rows 0..15) is the subset h in [32, 96) U [144, 176) U [192, 196).
__device__ __forceinline__ void halo_cell(int h, int &hr, int &hc)
{
    if (h < 128) {
        const int row = h >> 5;
        hr = row == 0 ? -2 : row == 1 ? -1 : row == 2 ? WJ : WJ + 1;
        hc = h & 31;
    } else if (h < 192) {
        const int col = (h - 128) >> 4;
        hc = col == 0 ? -2 : col == 1 ? -1 : col == 2 ? WK : WK + 1;
        hr = (h - 128) & 15;
    } else {
        const int q = h - 192;
        hr = (q & 1) ? WJ : -1;
        hc = (q & 2) ? WK : -1;
    }
}

__device__ __forceinline__ bool halo_has_velocity(int h)
{
    return (h >= 32 && h < 96) || (h >= 144 && h < 176) || (h >= 192 && h < NHALO);
}

// velocities of one cell of the state ring into the velocity rings
template <typename T, bool SST>
__device__ __forceinline__ void cell_prims(Smem<T> &s, int pl, int rr, int cc, T mu_pl, T mu_prev)
{
    const T *u = s.U[pl & 1][rr + 2][cc + 2];
    vel_rcp(u[0], u[1], u[2], u[3], s.R[pl % 3][rr + 1][cc + 1]);
    T dv[4];
    vdiv(u, dv);
    T *o = s.Dv[pl & 1][rr + 1][cc + 1];
    o[0] = dv[0]; o[1] = dv[1]; o[2] = dv[2]; o[3] = dv[3];
    if constexpr (!SST) o[4] = T(0.5) * (mu_pl + mu_prev);
}

template <typename T> __device__ __forceinline__ void store5(T *dst, const double *v)
{
#pragma unroll
    for (int q = 0; q < 5; q++) dst[q] = T(v[q]);
}

// The y sweep of ring cell (rr, cc) of plane slot q: hi (face above) and lo
// (face below), from the state ring.
template <typename T>
__device__ __forceinline__ void sweep_y(const Smem<T> &s, int q, int rr, int cc, T *hi, T *lo)
{
    CellC<T> c;
    const T *Uc = s.U[q][rr + 2][cc + 2];
#pragma unroll
    for (int v = 0; v < 5; v++) c.u[v] = Uc[v];
    cell_consts(c);
    const T *a1 = s.U[q][rr + 3][cc + 2], *b1 = s.U[q][rr + 1][cc + 2];
    T fw[5] = {a1[0], a1[2], a1[3], a1[1], a1[4]};
    T bw[5] = {b1[0], b1[2], b1[3], b1[1], b1[4]};
    recon_y(c, fw, bw, hi, lo);
}

template <typename T>
__device__ __forceinline__ void sweep_z(const Smem<T> &s, int q, int rr, int cc, T *hi, T *lo)
{
    CellC<T> c;
    const T *Uc = s.U[q][rr + 2][cc + 2];
#pragma unroll
    for (int v = 0; v < 5; v++) c.u[v] = Uc[v];
    cell_consts(c);
    const T *a1 = s.U[q][rr + 2][cc + 3], *b1 = s.U[q][rr + 2][cc + 1];
    T fw[5] = {a1[0], a1[3], a1[1], a1[2], a1[4]};
    T bw[5] = {b1[0], b1[3], b1[1], b1[2], b1[4]};
    recon_z(c, fw, bw, hi, lo);
}

// y flux of the face between ring rows rr and rr+1 at column cc, plane i
// (velocity slots: s0 plane i, sm1 plane i-1, sp1 plane i+1; u0 Dv of plane i)
template <typename T, bool SST>
__device__ __forceinline__ void face_y(const Smem<T> &s, const Consts &kc, int q0, int u0, int sm1, int s0, int sp1,
                                       int rr, int cc, const T *Lm, const T *Rp, T *F)
{
    const int a = rr + 1, b = cc + 1;
    const T *vm = s.Dv[u0][a][b], *vp = s.Dv[u0][a + 1][b];
    const T m_f = SST ? T(0.5) * (s.U[q0][rr + 3][cc + 2][0] + s.U[q0][rr + 2][cc + 2][0]) : vp[4];
    fused_face<T, 2, SST>(Lm, Rp, vm, vm[3], vp, vp[3], s.R[sp1][a + 1][b], s.R[sp1][a][b], s.R[sm1][a + 1][b],
                          s.R[sm1][a][b], s.R[s0][a + 1][b + 1], s.R[s0][a][b + 1], s.R[s0][a + 1][b - 1],
                          s.R[s0][a][b - 1], m_f, kc, F);
}

// z flux of the face between ring columns cc and cc+1 at row rr, plane i
template <typename T, bool SST>
__device__ __forceinline__ void face_z(const Smem<T> &s, const Consts &kc, int q0, int u0, int sm1, int s0, int sp1,
                                       int rr, int cc, const T *Lm, const T *Rp, T *F)
{
    const int a = rr + 1, b = cc + 1;
    const T *vm = s.Dv[u0][a][b], *vp = s.Dv[u0][a][b + 1];
    const T m_f = SST ? T(0.5) * (s.U[q0][rr + 2][cc + 3][0] + s.U[q0][rr + 2][cc + 2][0]) : vp[4];
    fused_face<T, 3, SST>(Lm, Rp, vm, vm[3], vp, vp[3], s.R[sp1][a][b + 1], s.R[sp1][a][b], s.R[sm1][a][b + 1],
                          s.R[sm1][a][b], s.R[s0][a + 1][b + 1], s.R[s0][a + 1][b], s.R[s0][a - 1][b + 1],
                          s.R[s0][a - 1][b], m_f, kc, F);
}

// The halo sweeps of plane p (warps 13, 14, 15; ring slot p & 1) into the
// buffers of p's parity: run for a segment's first plane in its prologue and
// for plane i+1 after plane i's stage combination, so the sweep phase before a
// plane's first barrier has the own sweeps only.  nyf, nzf: the y and z
// boundary-face array strides of the non-temporal setups.
template <typename T>
__device__ __forceinline__ void halo_sweeps(Smem<T> &s, const Args<T> &a, int p, int r, int l, int j0, int k0, int H,
                                            int D, long long nyf, long long nzf, bool tpl, bool ybot, bool ytop,
                                            bool zlft, bool zrgt)
{
    const int k = k0 + l;
    const int qp = p & 1;
    if (r == WJ - 3) {
        // halo row -1: its state on the face above (the tile's bottom faces)
        if (k <= D && (ybot || !tpl)) { // temporal bottom boundary: row 0's own state, below
            T hb[5], tmp[5];
            if (ybot) {
                sweep_y(s, qp, -1, l, hb, tmp);
            } else {
                const long long fo = (long long)(p - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) hb[q] = a.bf.y0[q * nyf + FSL_FACE(fo, nyf)];
            }
#pragma unroll
            for (int q = 0; q < 5; q++) s.HyB[qp][l][q] = hb[q];
        }
    } else if (r == WJ - 2) {
        // halo row 16: its state on the face below (the tile's top
        // faces), or the top boundary's outer state when row 16 is
        // the ghost row
        if (k <= D) {
            if (ytop) {
                T lo[5], tmp[5];
                sweep_y(s, qp, WJ, l, tmp, lo);
#pragma unroll
                for (int q = 0; q < 5; q++) s.LoH[qp][l][q] = lo[q];
            } else if (j0 + WJ == H + 1 && !tpl) {
                const long long fo = (long long)(p - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) s.LoH[qp][l][q] = a.bf.yH[q * nyf + FSL_FACE(fo, nyf)];
            }
        }
    } else if (r == WJ - 1) {
        // halo columns -1 (lanes 0..15) and 32 (lanes 16..31): one
        // sweep for the whole warp, each half on its own column
        const int rr = l & 15, jr = j0 + rr;
        const bool left = l < 16;
        const bool act = jr <= H && (left || k0 + WK - 1 <= D);
        // periodic z: ghost column -1 holds cell DEP, ghost column 32 cell 1
        const bool ring = left ? (zlft || tpl) : (zrgt || tpl);
        // the left half keeps the state on the face beyond its column,
        // the right half the state on the face before its column
        T o[5];
        if (act && ring) {
            T hv[5], lv[5];
            sweep_z(s, qp, rr, left ? -1 : WK, hv, lv);
#pragma unroll
            for (int q = 0; q < 5; q++) o[q] = left ? hv[q] : lv[q];
        } else if (act) {
            const long long fo = (long long)(p - 1) * H + (jr - 1);
            const T *bfz = left ? a.bf.z0 : a.bf.zD;
#pragma unroll
            for (int q = 0; q < 5; q++) o[q] = bfz[q * nzf + FSL_FACE(fo, nzf)];
        }
        if (act) {
            T *dst = left ? s.HzL[qp][rr] : s.LzR[qp][rr];
#pragma unroll
            for (int q = 0; q < 5; q++) dst[q] = o[q];
        }
    }
}

// Block b of a domain's stage launch of nb blocks: its share of the
// (tile, plane) pairs, and with a.co the Courant maximum of what it wrote.
template <typename T, bool SST>
__device__ __forceinline__ void wide_block(Smem<T> &s, const Grid &g, const Consts &kc, const Args<T> &a, int b,
                                           int nb)
{
    const int L = g.L, H = g.H, D = g.D;
    const int t = threadIdx.x, r = t >> 5, l = t & 31;
    const long long fs = g.fstride;
    const double *__restrict__ cu = a.cur;
    const T *__restrict__ mu = a.mu;
    const long long nxf = (long long)H * D, nyf = (long long)L * D, nzf = (long long)L * H;
    const double dtx = a.ds->dtx, dty = a.ds->dty, dtz = a.ds->dtz;
    const double one_third = 1. / 3., two_thirds = 2. / 3.;
    // temporal setup: the boundary faces' outer states are formed here from
    // the state itself (the periodic x and z rules and the zero-gradient y
    // rule of the boundary pass), and every boundary cell written also fills
    // the ghost cells that copy it, so no ghost-fill or boundary pass runs
    // between the stages
    const bool tpl = kc.setup == FSL_SETUP_TEMPORAL;
    // this thread's halo cell (threads 0..195)
    int hr = 0, hc = 0;
    const bool hthread = t < NHALO;
    if (hthread) halo_cell(t, hr, hc);
    const bool hvel = hthread && halo_has_velocity(t);
    s.comax[r][l] = 0.0;

    const int ntk = (D + WK - 1) / WK, ntj = (H + WJ - 1) / WJ;
    const long long ntiles = (long long)ntk * ntj, total = ntiles * L;
    // heads: planes 1..Hd of every tile; tails: planes Hd+1..L of every tile.
    // With more blocks than tiles, block b < ntiles takes the head of tile b
    // and the other blocks share the tails; a tail plane counts 1.03 head
    // planes (the tail blocks start several segments, each with a prologue,
    // and run out of step with their neighbours), so the heads are a little
    // longer.  Measured at 512x256x256 per stage launch: 2.404, 2.373, 2.349,
    // 2.357, 2.362 ms for weights 1.00, 1.01, 1.03, 1.06, 1.09.
    long long Hd, pos, end;
    if (nb > ntiles) {
        Hd = min((long long)L, (103LL * ntiles * L) / (100LL * (nb - ntiles) + 103LL * ntiles));
        const long long tails = ntiles * (L - Hd), nt = nb - ntiles;
        pos = b < ntiles ? b * Hd : ntiles * Hd + tails * (b - ntiles) / nt;
        end = b < ntiles ? (b + 1) * Hd : ntiles * Hd + tails * (b - ntiles + 1) / nt;
    } else {
        Hd = min((long long)L, total / nb);
        pos = total * b / nb;
        end = total * (b + 1) / nb;
    }
    const long long Lt = L - Hd, nhead = ntiles * Hd;
    while (pos < end) {
        long long tile, run;
        int i0;
        if (pos < nhead) {
            tile = pos / Hd;
            i0 = (int)(pos % Hd) + 1;
            run = Hd - (pos % Hd);
        } else {
            const long long v = pos - nhead;
            tile = v / Lt;
            i0 = (int)(Hd + v % Lt) + 1;
            run = Lt - (v % Lt);
        }
        const int i1 = i0 + (int)min(run, end - pos) - 1;
        pos += i1 - i0 + 1;
        const int k0 = (int)(tile % ntk) * WK + 1, j0 = (int)(tile / ntk) * WJ + 1;
        const int j = j0 + r, k = k0 + l;
        // temporal setup (periodic z): the ring's columns beyond the ghost
        // columns, k = -1 and k = DEP+2, hold cells DEP-1 and 2, so the z
        // boundary faces' outer states are sweeps over the ring like any
        // other face's
        const int kmin = tpl ? -1 : 0, kmax = tpl ? D + 2 : D + 1;
        const bool own = j <= H && k <= D;               // interior cell of this thread
        const bool live = j <= H + 1 && k <= kmax;       // cell in the padded array (or its periodic image)
        const long long cj = g.idx(0, j, k == D + 2 ? 2 : k);
        // halo cell of this thread (padded indices)
        const int hj = j0 + hr, hk = k0 + hc;
        const bool hlive = hthread && hj >= 0 && hj <= H + 1 && hk >= kmin && hk <= kmax;
        const bool hvlive = hvel && hlive;
        const long long hcj = g.idx(0, hj, hk == -1 ? D - 1 : hk == D + 2 ? 2 : hk);
        const bool ybot = j0 > 1, ytop = j0 + WJ <= H, zlft = k0 > 1, zrgt = k0 + WK <= D;

        T hix[5], Fxp[5];
#pragma unroll
        for (int q = 0; q < 5; q++) hix[q] = Fxp[q] = T(0.);
        T mu0 = 0, mu1 = 0, mu2 = 0, hmu0 = 0, hmu1 = 0, hmu2 = 0;
        double pown[5], phal[5], base[5], unv[5];
#pragma unroll
        for (int q = 0; q < 5; q++) pown[q] = phal[q] = base[q] = unv[q] = 0.;

        __syncthreads(); // the previous segment's readers of the rings are done
        // ---- prologue: planes i0, i0+1 into the state ring, velocities of
        // planes i0-1 .. i0+1, the flux of face i0 - 1/2 ----
        {
#pragma unroll
            for (int p = 0; p < 2; p++) {
                const int pl = i0 + p;
                if (live && pl <= L + 1) {
                    load5(cu, fs, cj + (long long)pl * g.pi, pown);
                    store5(s.U[pl & 1][r + 2][l + 2], pown);
                }
                if (hlive && pl <= L + 1) {
                    load5(cu, fs, hcj + (long long)pl * g.pi, phal);
                    store5(s.U[pl & 1][hr + 2][hc + 2], phal);
                }
            }
            T Um[5] = {0, 0, 0, 0, 0}, mum = 0, hmum = 0;
            if (live) {
                load5(cu, fs, cj + (long long)(i0 - 1) * g.pi, Um);
                vel_rcp(Um[0], Um[1], Um[2], Um[3], s.R[(i0 - 1) % 3][r + 1][l + 1]);
                if constexpr (!SST) {
                    mum = mu[FSL_CELL(cj + (long long)(i0 - 1) * g.pi, fs)];
                    mu0 = mu[FSL_CELL(cj + (long long)i0 * g.pi, fs)];
                    mu1 = mu[FSL_CELL(cj + (long long)(i0 + 1) * g.pi, fs)];
                }
                cell_prims<T, SST>(s, i0, r, l, mu0, mum);
                cell_prims<T, SST>(s, i0 + 1, r, l, mu1, mu0);
            }
            if (hvlive) {
                T Hm[5];
                load5(cu, fs, hcj + (long long)(i0 - 1) * g.pi, Hm);
                vel_rcp(Hm[0], Hm[1], Hm[2], Hm[3], s.R[(i0 - 1) % 3][hr + 1][hc + 1]);
                if constexpr (!SST) {
                    hmum = mu[FSL_CELL(hcj + (long long)(i0 - 1) * g.pi, fs)];
                    hmu0 = mu[FSL_CELL(hcj + (long long)i0 * g.pi, fs)];
                    hmu1 = mu[FSL_CELL(hcj + (long long)(i0 + 1) * g.pi, fs)];
                }
                cell_prims<T, SST>(s, i0, hr, hc, hmu0, hmum);
                cell_prims<T, SST>(s, i0 + 1, hr, hc, hmu1, hmu0);
            }
            __syncthreads();
            if (r >= WJ - 3) halo_sweeps(s, a, i0, r, l, j0, k0, H, D, nyf, nzf, tpl, ybot, ytop, zlft, zrgt);
            if (own) {
                T hm[5], lo[5], hin[5], dm[4], tmp[5];
                const T *Uc = s.U[i0 & 1][r + 2][l + 2], *Un = s.U[(i0 + 1) & 1][r + 2][l + 2];
                {
                    CellC<T> cc;
#pragma unroll
                    for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
                    cell_consts(cc);
                    recon_x(cc, Un, Um, hin, lo);
                }
                if (i0 == 1 && tpl) {
                    recon_at<T, 0>(g, cu, g.idx(L, j, k), hm, tmp); // periodic x: cell LEN's face
                } else if (i0 == 1) {
                    const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
                    for (int q = 0; q < 5; q++) hm[q] = a.bf.x0[q * nxf + FSL_FACE(fo, nxf)];
                } else {
                    recon_at<T, 0>(g, cu, cj + (long long)(i0 - 1) * g.pi, hm, tmp);
                }
                vdiv(Um, dm);
                const T *dc = s.Dv[i0 & 1][r + 1][l + 1];
                const int sb = (i0 - 1) % 3, sf = i0 % 3;
                const T m_f = SST ? T(0.5) * (Uc[0] + Um[0]) : dc[4];
                fused_face<T, 1, SST>(hm, lo, dm, dm[3], dc, dc[3], s.R[sf][r + 2][l + 1], s.R[sb][r + 2][l + 1],
                                      s.R[sf][r][l + 1], s.R[sb][r][l + 1], s.R[sf][r + 1][l + 2],
                                      s.R[sb][r + 1][l + 2], s.R[sf][r + 1][l], s.R[sb][r + 1][l], m_f, kc, Fxp);
#pragma unroll
                for (int q = 0; q < 5; q++) hix[q] = hin[q];
            }
        }

        for (int i = i0; i <= i1; i++) {
            const int sm1 = (i + 2) % 3, s0 = i % 3, sp1 = (i + 1) % 3;
            const int q0 = i & 1, q1 = (i + 1) & 1;
            // (a) plane i+2 in flight; the FP64 operands of the combination
            if (live && i + 2 <= L + 1) load5(cu, fs, cj + (long long)(i + 2) * g.pi, pown);
            if (hlive && i + 2 <= L + 1) load5(cu, fs, hcj + (long long)(i + 2) * g.pi, phal);
            if (own) {
                const long long c = FSL_CELL(cj + (long long)i * g.pi, fs);
#pragma unroll
                for (int q = 0; q < 5; q++) base[q] = cu[q * fs + c];
                if (a.stage != 1) {
#pragma unroll
                    for (int q = 0; q < 5; q++) unv[q] = a.un[q * fs + c];
                }
            }
            if constexpr (!SST) {
                if (live && i + 2 <= L + 1) mu2 = mu[FSL_CELL(cj + (long long)(i + 2) * g.pi, fs)];
                if (hvlive && i + 2 <= L + 1) hmu2 = mu[FSL_CELL(hcj + (long long)(i + 2) * g.pi, fs)];
            }
            // (b) y and z sweeps of the own cell, the boundary outer states,
            // and the halo sweeps (warps 13..15)
            T hy[5], hz[5], lz[5];
#pragma unroll
            for (int q = 0; q < 5; q++) hy[q] = hz[q] = lz[q] = T(0.);
            if (own) {
                CellC<T> cc;
                const T *Uc = s.U[q0][r + 2][l + 2];
#pragma unroll
                for (int q = 0; q < 5; q++) cc.u[q] = Uc[q];
                cell_consts(cc);
                T lo[5];
                {
                    const T *a1 = s.U[q0][r + 3][l + 2], *b1 = s.U[q0][r + 1][l + 2];
                    T fw[5] = {a1[0], a1[2], a1[3], a1[1], a1[4]};
                    T bw[5] = {b1[0], b1[2], b1[3], b1[1], b1[4]};
                    recon_y(cc, fw, bw, hy, lo);
                }
#pragma unroll
                for (int q = 0; q < 5; q++) s.Lo[r][l][q] = lo[q];
                {
                    const T *a1 = s.U[q0][r + 2][l + 3], *b1 = s.U[q0][r + 2][l + 1];
                    T fw[5] = {a1[0], a1[3], a1[1], a1[2], a1[4]};
                    T bw[5] = {b1[0], b1[3], b1[1], b1[2], b1[4]};
                    recon_z(cc, fw, bw, hz, lz);
                }
                if (l == 0) {
#pragma unroll
                    for (int q = 0; q < 5; q++) s.Lz0[r][q] = lz[q];
                }
            } else if (j == H + 1 && k <= D && !tpl) {
                // the face below this ghost row: the top boundary's outer state
                const long long fo = (long long)(i - 1) * D + (k - 1);
#pragma unroll
                for (int q = 0; q < 5; q++) s.Lo[r][l][q] = a.bf.yH[q * nyf + FSL_FACE(fo, nyf)];
            } else if (k == D + 1 && j <= H) {
                // beyond the last column: the far z boundary's outer state (shuffled to lane l-1)
                if (tpl) {
                    T tz[5];
                    sweep_z(s, q0, r, l, tz, lz); // periodic z: this ghost column holds cell 1
                } else {
                    const long long fo = (long long)(i - 1) * H + (j - 1);
#pragma unroll
                    for (int q = 0; q < 5; q++) lz[q] = a.bf.zD[q * nzf + FSL_FACE(fo, nzf)];
                }
            }
            __syncthreads();
            // (c) the own faces: y above, z beyond, x ahead; the tile's bottom
            // y faces (warp 12) and left z faces (warp 11)
            T Fz[5], Fx[5], hin[5];
#pragma unroll
            for (int q = 0; q < 5; q++) Fz[q] = Fx[q] = hin[q] = T(0.);
            {
                T lzn[5];
#pragma unroll
                for (int q = 0; q < 5; q++) lzn[q] = __shfl_down_sync(0xffffffffu, lz[q], 1);
                if (own) {
                    if (l == WK - 1) {
#pragma unroll
                        for (int q = 0; q < 5; q++) lzn[q] = s.LzR[q0][r][q];
                    }
                    face_z<T, SST>(s, kc, q0, q0, sm1, s0, sp1, r, l, hz, lzn, Fz);
                    T F[5];
                    // the state above the face: row r+1's (the halo row's for
                    // row 15); at the temporal top boundary the cell's own
                    T up[5];
                    {
                        const T *src = r + 1 < WJ ? s.Lo[r + 1][l] : s.LoH[q0][l];
#pragma unroll
                        for (int q = 0; q < 5; q++) up[q] = (tpl && j == H) ? hy[q] : src[q];
                    }
                    face_y<T, SST>(s, kc, q0, q0, sm1, s0, sp1, r, l, hy, up, F);
#pragma unroll
                    for (int q = 0; q < 5; q++) s.Fy[r + 1][l][q] = F[q];
                }
            }
            if (r == WJ - 4 && k <= D && j0 <= H) {
                T F[5];
                face_y<T, SST>(s, kc, q0, q0, sm1, s0, sp1, -1, l, (tpl && !ybot) ? s.Lo[0][l] : s.HyB[q0][l], s.Lo[0][l],
                               F);
#pragma unroll
                for (int q = 0; q < 5; q++) s.Fy[0][l][q] = F[q];
            }
            if (r == WJ - 5 && l < WJ && j0 + l <= H && k0 <= D) {
                T F[5];
                face_z<T, SST>(s, kc, q0, q0, sm1, s0, sp1, l, -1, s.HzL[q0][l], s.Lz0[l], F);
#pragma unroll
                for (int q = 0; q < 5; q++) s.FzL[l][q] = F[q];
            }
            if (own) {
                T lo[5];
                if (i + 1 <= L) {
                    CellC<T> cc;
                    const T *Un = s.U[q1][r + 2][l + 2];
#pragma unroll
                    for (int q = 0; q < 5; q++) cc.u[q] = Un[q];
                    cell_consts(cc);
                    T fw2[5];
#pragma unroll
                    for (int q = 0; q < 5; q++) fw2[q] = T(pown[q]);
                    recon_x(cc, fw2, s.U[q0][r + 2][l + 2], hin, lo);
                } else if (tpl) {
                    T tx[5];
                    recon_at<T, 0>(g, cu, g.idx(1, j, k), tx, lo); // periodic x: cell 1's face
                } else {
                    const long long fo = (long long)(j - 1) * D + (k - 1);
#pragma unroll
                    for (int q = 0; q < 5; q++) lo[q] = a.bf.xL[q * nxf + FSL_FACE(fo, nxf)];
                }
                const T *dc = s.Dv[q0][r + 1][l + 1], *dn = s.Dv[q1][r + 1][l + 1];
                const T m_f = SST ? T(0.5) * (s.U[q1][r + 2][l + 2][0] + s.U[q0][r + 2][l + 2][0]) : dn[4];
                fused_face<T, 1, SST>(hix, lo, dc, dc[3], dn, dn[3], s.R[sp1][r + 2][l + 1], s.R[s0][r + 2][l + 1],
                                      s.R[sp1][r][l + 1], s.R[s0][r][l + 1], s.R[sp1][r + 1][l + 2],
                                      s.R[s0][r + 1][l + 2], s.R[sp1][r + 1][l], s.R[s0][r + 1][l], m_f, kc, Fx);
            }
            T Fzm[5];
#pragma unroll
            for (int q = 0; q < 5; q++) Fzm[q] = __shfl_up_sync(0xffffffffu, Fz[q], 1);
            __syncthreads();
            // (d) divergence and stage combination (src/evolution.c:29-161):
            // the divergence in FP32, the combination in FP64
            if (own) {
                if (l == 0) {
#pragma unroll
                    for (int q = 0; q < 5; q++) Fzm[q] = s.FzL[r][q];
                }
                const long long c = FSL_CELL(cj + (long long)i * g.pi, fs);
#pragma unroll
                for (int q = 0; q < 5; q++) {
                    const T X = T(dtx) * (Fxp[q] - Fx[q]);
                    const T Y = T(dty) * (s.Fy[r][l][q] - s.Fy[r + 1][l][q]);
                    const T Z = T(dtz) * (Fzm[q] - Fz[q]);
                    const double inc = (double)(X + Y + Z);
                    double o;
                    if (a.stage == 1) o = base[q] + inc;
                    else if (a.stage == 2) o = 0.75 * unv[q] + 0.25 * (base[q] + inc);
                    else o = one_third * unv[q] + two_thirds * (base[q] + inc);
                    a.out[q * fs + c] = o;
                    base[q] = o;
                }
                // the FP32 velocities of the closure's features (rho u as
                // float times the float of the FP64 reciprocal)
                float vu = 0.f, vv = 0.f, vw = 0.f;
                // 1/rho of the written cell, shared by the velocities and the
                // acoustic Courant number (the last stage only)
                const double ir = (a.vel || a.co) ? 1. / base[0] : 0.;
                if (a.vel) {
                    const float rr = (float)ir;
                    vu = (float)base[1] * rr;
                    vv = (float)base[2] * rr;
                    vw = (float)base[3] * rr;
                    a.vel[c] = vu;
                    a.vel[fs + c] = vv;
                    a.vel[2 * fs + c] = vw;
                }
                const bool bx = i == 1 || i == L, by = j == 1 || j == H, bz = k == 1 || k == D;
                if (tpl && bz && !(bx || by)) {
                    // the one ghost cell that copies a z-edge cell (periodic z)
                    const long long gc = FSL_CELL(c + ((k == D ? 0 : D + 1) - k), fs);
#pragma unroll
                    for (int q = 0; q < 5; q++) a.out[q * fs + gc] = base[q];
                    if (a.vel) {
                        a.vel[gc] = vu;
                        a.vel[fs + gc] = vv;
                        a.vel[2 * fs + gc] = vw;
                    }
                } else if (tpl && (bx || by || bz)) {
                    // the ghost cells that copy this cell (the ghost pass's
                    // periodic x and z and zero-gradient y rules, edges and
                    // corners included)
                    const int xi[2] = {i, i == L ? 0 : (i == 1 ? L + 1 : -1)};
                    const int yj[2] = {j, j == 1 ? 0 : (j == H ? H + 1 : -1)};
                    const int zk[2] = {k, k == D ? 0 : (k == 1 ? D + 1 : -1)};
#pragma unroll
                    for (int e = 1; e < 8; e++) {
                        const int gi = xi[e & 1], gj = yj[(e >> 1) & 1], gk = zk[e >> 2];
                        if (gi < 0 || gj < 0 || gk < 0) continue;
                        const long long gc = FSL_CELL(g.idx(gi, gj, gk), fs);
#pragma unroll
                        for (int q = 0; q < 5; q++) a.out[q * fs + gc] = base[q];
                        if (a.vel) {
                            a.vel[gc] = vu;
                            a.vel[fs + gc] = vv;
                            a.vel[2 * fs + gc] = vw;
                        }
                    }
                }
                if (a.co && i >= a.co_i0 && i <= a.co_i1) {
                    const double Co =
                        cell_courant_ir(kc.cfl_mode, base[0], ir, base[1], base[2], base[3], base[4], dtx, dty, dtz);
                    const double m = s.comax[r][l];
                    s.comax[r][l] = (Co > m) ? Co : m;
                    if (!(base[0] > 0.0)) atomicOr(a.status, 2u);
                }
            }
            // the next plane's halo sweeps (its state is in the ring)
            if (r >= WJ - 3 && i < i1)
                halo_sweeps(s, a, i + 1, r, l, j0, k0, H, D, nyf, nzf, tpl, ybot, ytop, zlft, zrgt);
            // (e) plane i+2 into the state ring slot of plane i and its
            // velocities into the slots of planes i-1 (reciprocal) and i
            // (division); advance the march
            if (i < i1) {
                if (live && i + 2 <= L + 1) {
                    store5(s.U[q0][r + 2][l + 2], pown);
                    cell_prims<T, SST>(s, i + 2, r, l, mu2, mu1);
                }
                if (hlive && i + 2 <= L + 1) {
                    store5(s.U[q0][hr + 2][hc + 2], phal);
                    if (hvel) cell_prims<T, SST>(s, i + 2, hr, hc, hmu2, hmu1);
                }
            }
#pragma unroll
            for (int q = 0; q < 5; q++) {
                Fxp[q] = Fx[q];
                hix[q] = hin[q];
            }
            mu0 = mu1;
            mu1 = mu2;
            hmu0 = hmu1;
            hmu1 = hmu2;
        }
    }
    if (a.co) {
        __syncthreads();
        double m = s.comax[r][l];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double x = __shfl_xor_sync(0xffffffffu, m, o);
            m = (x > m) ? x : m;
        }
        __syncthreads();
        if (l == 0) s.comax[r][0] = m;
        __syncthreads();
        if (t == 0) {
            m = 0.0;
#pragma unroll
            for (int q = 0; q < WJ; q++) m = (s.comax[q][0] > m) ? s.comax[q][0] : m;
            // non-negative doubles order like their bit patterns
            atomicMax(a.co, (unsigned long long)__double_as_longlong(m));
        }
        __syncthreads(); // comax is reset by the next block's work
    }
}

// One domain of a (multi-domain) persistent stage launch: its grid, constants
// and buffers.  Stage s reads st[s-1] and writes out[s-1] (U -> Up -> Uq -> U);
// nb is the number of blocks of the domain's own launch, whose split of the
// (tile, plane) pairs a multi-domain launch keeps, so a domain's results do
// not depend on the other domains it is stepped with.
struct WideMember {
    Grid g;
    Consts kc;
    const double *st[3];
    double *out[3];
    const double *un;
    const float *mu;
    BF<float> bf;
    const DevScalars *ds;
    unsigned long long *co; // stage 3 Courant maximum (device scalar)
    unsigned int *status;
    int co_i0, co_i1;
    int nb;
    int setup, BL_HIG;
    Disturb dist;
    float *vel; // stage 3 also writes the FP32 velocities of its output (null: no)
};

// A grid-wide barrier with a bounded wait: false (and *err set) when the
// other blocks did not all arrive within `limit` polls.  Only for launches
// whose blocks are all resident (cooperative launches).
struct GridBarrier {
    unsigned *count, *gen;
    int *err;
    unsigned limit;
};

__device__ __forceinline__ bool grid_sync(const GridBarrier &gb, unsigned nblocks)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = gb.gen;
        const unsigned g0 = *gen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(gb.count, 1u) + 1u == nblocks) {
            atomicExch(gb.count, 0u);
            __threadfence();
            atomicAdd(gb.gen, 1u);
        } else {
            unsigned n = 0;
            while (*gen == g0) {
                if (++n > gb.limit) {
                    ok = 0;
                    atomicExch(gb.err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_s = ok && *(volatile int *)gb.err == 0;
    }
    __syncthreads();
    return ok_s != 0;
}

// The work of one persistent launch: stages s_begin .. s_end of nmem domains
// (m0 alone when mem is null).  With items, block x runs the (domain, block)
// pairs items[start[x] .. start[x+1]); without, block x is block x of the
// single domain.  Between two stages of one launch the blocks meet at a grid
// barrier (the temporal setup's stages write their own ghost cells and form
// their boundary states), so a whole step of many domains is one launch.
struct WideWork {
    WideMember m0;
    const WideMember *mem;
    int nmem;
    const int2 *items;
    const int *start;
    int s_begin, s_end;
    int courant; // stage 3 accumulates the Courant maximum
    GridBarrier bar;
};

__device__ __forceinline__ Args<float> member_args(const WideMember &M, int st, bool courant)
{
    Args<float> a;
    a.cur = M.st[st - 1];
    a.un = M.un;
    a.out = M.out[st - 1];
    a.mu = M.mu;
    a.bf = M.bf;
    a.ds = M.ds;
    a.co = (st == 3 && courant) ? M.co : nullptr;
    a.co_i0 = M.co_i0;
    a.co_i1 = M.co_i1;
    a.status = M.status;
    a.stage = st;
    a.seg = 0;
    a.vel = st == 3 ? M.vel : nullptr;
    return a;
}

// MULTI = false: one stage of the domain w.m0, block x its block x (its
// descriptor stays in the parameter space).  MULTI = true: the work list.
// Both instantiate the same block code (wide_block), so a domain stepped
// alone and in a multi-domain launch computes the same values.
template <bool SST, bool MULTI>
__global__ void __launch_bounds__(NT, 1) k_wide(WideWork w)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem<float> &s = *reinterpret_cast<Smem<float> *>(smraw);
    if constexpr (!MULTI) {
        wide_block<float, SST>(s, w.m0.g, w.m0.kc, member_args(w.m0, w.s_begin, w.courant != 0), blockIdx.x,
                               w.m0.nb);
    } else {
        for (int st = w.s_begin; st <= w.s_end; st++) {
            const int i0 = w.start[blockIdx.x], i1 = w.start[blockIdx.x + 1];
            for (int it = i0; it < i1; it++) {
                const int2 x = w.items[it];
                const int mi = x.x, b = x.y;
                // the member's descriptor and stage arguments in shared memory:
                // the block code reads them where it needs them instead of
                // holding them in registers
                __shared__ WideMember sm;
                __shared__ Args<float> sa;
                __syncthreads(); // the previous item's readers are done
                if (threadIdx.x == 0) {
                    sm = w.mem[mi];
                    sa = member_args(sm, st, w.courant != 0);
                }
                __syncthreads();
                wide_block<float, SST>(s, sm.g, sm.kc, sa, b, sm.nb);
            }
            if (st == w.s_end) break;
            // the stage's outputs (ghost cells included) complete before the next reads them
            if (!grid_sync(w.bar, gridDim.x)) return;
    }
    }
}

// Blocks of the persistent grid: one per SM, fewer when the domain has fewer
// than 16 planes of tiles per SM (each block then marches at least that far).
// 32 planes measured slower for small domains stepped alone (8.4e8 against
// 1.33e9 cell-stage updates/s over the 32 ensemble layers one by one).
inline int wide_blocks(const Grid &g, int sms)
{
    const long long ntiles = (long long)((g.D + WK - 1) / WK) * ((g.H + WJ - 1) / WJ);
    const long long units = ntiles * g.L;
    const long long want = (units + 15) / 16;
    return (int)std::max(1LL, std::min((long long)sms, want));
}

// The single-domain member descriptor of a context (FP32 buffers).
inline WideMember wide_member(const Ctx &c, const float *mu, BF<float> bf, int sms)
{
    WideMember m;
    m.g = c.g;
    m.kc = c.k;
    m.st[0] = c.U; m.st[1] = c.Up; m.st[2] = c.Uq;
    m.out[0] = c.Up; m.out[1] = c.Uq; m.out[2] = c.U;
    m.un = c.U;
    m.mu = mu;
    m.bf = bf;
    m.ds = c.ds;
    m.co = &c.ds->co_bits;
    m.status = &c.ds->status;
    m.co_i0 = c.co_i0;
    m.co_i1 = c.co_i1;
    m.nb = wide_blocks(c.g, sms);
    m.setup = c.k.setup;
    m.BL_HIG = c.k.BL_HIG;
    m.dist = c.dist;
    m.vel = nullptr;
    return m;
}

template <bool SST, bool MULTI> inline bool wide_attr()
{
    static std::atomic<uint64_t> attr{0};
    return smem_limit_once((const void *)k_wide<SST, MULTI>, sizeof(Smem<float>), attr);
}

// One stage of one domain (the FP32 bulk's fused stage with the reference
// reconstruction).  The buffers are the context's fixed stage sequence.
template <bool SST>
int launch_wide(Ctx &c, int stage, const double *cur, const double *un, double *out, const float *mu,
                BF<float> bf, bool courant, float *vel)
{
    (void)cur; (void)un; (void)out; // always U -> Up -> Uq -> U with U^n = U
    if (!wide_attr<SST, false>()) return -1;
    WideWork w{};
    w.m0 = wide_member(c, mu, bf, c.sms);
    w.m0.vel = vel;
    w.mem = nullptr;
    w.nmem = 1;
    w.items = nullptr;
    w.start = nullptr;
    w.s_begin = w.s_end = stage;
    w.courant = courant ? 1 : 0;
    prof_begin(c, FSL_K_STAGE);
    k_wide<SST, false><<<w.m0.nb, NT, sizeof(Smem<float>), c.stream>>>(w);
    prof_end(c, FSL_K_STAGE, 1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

} // namespace wide
} // namespace fsl
