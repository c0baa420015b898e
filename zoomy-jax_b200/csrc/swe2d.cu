// Cartesian 2-D shallow-water finite-volume step for sm_100a.
//
// One stage = one explicit stage of zoomy_jax's flux operator fused with the
// Shu-Osher update (zoomy_jax/fvm/solver_jax.py:722-895 and 990-1074;
// zoomy_jax/fvm/solver2/blocks.py:129-287, march.py:126-157):
//
//   halo load -> W = (b, eta, u, v) or (b, h, qx, qy) -> LSQ gradient (3x3
//   least-squares stencil, boundary ghosts) -> neighbour bounds -> limiter ->
//   tied / demoted slopes -> face traces with the Audusse clip -> Rusanov or
//   hydrostatic-reconstruction HLL face flux, each face once per tile ->
//   divergence + cell-edge bed source -> Q_out = a Q0 + (1 - a)(Qk + b dt L).
//
// Data layout: SoA planes (the reference's (n_state, n_cells) layout), cell
// (i, j) at i*ny + j.  Two kernels implement a stage.  The tile kernel
// (swe2d_stage_kernel): a CTA owns a TX x 32 tile (32 cells along the
// contiguous y axis = one warp-wide coalesced row) and stages the tile plus a
// 2-cell halo in shared memory; every face of the tile is evaluated exactly
// once -- the generic stage API, first order, and the frame of grids with a
// periodic side.  The strip kernel (swe2d_strip_kernel): one warp marches a
// 32-column strip down its rows in registers -- the fused step (interior and
// boundary launches side by side).  The final stage also folds in Manning
// friction, the troubled-cell flag and the float64 maximum wave speed that
// sets the next dt, so a step queues with no host synchronisation.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace zb {

constexpr int TY = 32;        // tile cells along y (contiguous)
constexpr int NT = 256;       // threads per CTA

template <typename T>
struct LsqTable {
  // [class 0..8][direction][slot]; slot 0..7 = the 3x3 neighbours (a, b) in
  // row-major order without (0, 0), 8 = x-boundary ghost, 9 = y-boundary ghost
  T w[9][2][10];
};

template <typename T>
struct SweParams {
  int nx, ny;
  T half_dx, half_dy;       // |face centre - cell centre|
  T kx, ky;                 // |face| / |cell| for x- and y-faces
  T g, eps_kp, eps_wet, manning_n;
  T vk_eps2;                // Venkatakrishnan eps^2
  int bc[4];                // left, right, bottom, top
  int limiter;
  int implicit_source;
  double cfl2r;             // cfl * 2 * r_in
  double den_fac;           // d * (2k + 1)
  double dt_max, t_end;
  double alpha, beta;       // Shu-Osher coefficients (generic stage)
  double dt_stage;          // generic stage: dt (< 0: read ctrl->dt)
  T inv6dx, inv6dy;         // interior least-squares gradient factors
  T inv4dx, inv4dy;         // 1 / (4 dx), 1 / (4 dy): side-class closed forms
  // output region of the strip kernel ([fast_i0, fast_i1) x [fast_j0,
  // fast_j1), empty when fast_i0 >= fast_i1); the tile kernel leaves these
  // cells alone
  int fast_i0, fast_i1, fast_j0, fast_j1;
  // 1: the strip region is the whole grid (fast_i0 = fast_j0 = 0; the strips
  // reach the boundary and keep the control block; no tile launch)
  int strip_full;
  // the bed's interior gradient and limiter value (planes gx, gy, phi of
  // zb_swe2d_bed_prepare), read by the eta / HLL-HR interior strip body;
  // nullptr: evaluated from b like every other variable
  const T* bed;
  LsqTable<T> lsq;
};

enum { MODE_STEP1 = 0, MODE_STEP2 = 1, MODE_EULER = 2, MODE_STAGE = 3 };

template <typename T, int TX>
struct Smem {
  static constexpr int R2X = TX + 4, R2Y = TY + 4, N2 = R2X * R2Y;
  static constexpr int R1X = TX + 2, R1Y = TY + 2, N1 = R1X * R1Y;
  static constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1);
  T b[N2], h[N2], w1[N2], w2[N2], w3[N2], aux[N2];
  T sx[4][N1], sy[4][N1];
  T fxh[NFX], fxt[NFX], fxl[NFX], fxr[NFX];
  T fyh[NFY], fyt[NFY], fyl[NFY], fyr[NFY];
};

// ── dt from the phase slot (solver2/blocks.py:64-95) ────────────────────────
__device__ __forceinline__ double dt_from_amax(double amax, double t,
                                               double cfl2r, double den_fac,
                                               double dt_max, double t_end) {
  double dt = cfl2r / (den_fac * amax);   // amax = 0 -> +inf, drops out
  dt = nmin(dt, dt_max);
  dt = nmin(dt, t_end - t);
  return dt;
}

// ── limiter candidates (reconstruction_jax.py:603-691) ──────────────────────
// Minmod / Barth-Jespersen on a Cartesian cell.  The four faces carry the
// increments +a, -a (x) and +c, -c (y).  With dpos = umax - u >= 0 and
// dneg = umin - u <= 0 a face with increment d > eps gives clip(dpos / d) and
// one with d < -eps gives clip(dneg / d) = clip(-dneg / |d|).  IEEE division
// is monotone in both operands, so the minimum over the four faces is exactly
// clip(min(dpos, -dneg) / max(|a|, |c|)) whenever max(|a|, |c|) > eps (a pair
// with |d| <= eps contributes 1 and never the minimum), and 1 otherwise: one
// division per variable instead of four, bit-identical to the per-face form in
// float64 (float32 divides with adiv, within its 2 ulp of that form).
template <typename T>
__device__ __forceinline__ T phi_clipmin(T a, T c, T dpos, T dneg) {
  const T m = fmx(fabs(a), fabs(c));
  const T dm = fmn(dpos, -dneg);
  const T r = clip01(adiv(dm, m));
  return m > T(1e-30) ? r : T(1);
}

template <typename T>
__device__ __forceinline__ T vk_cand(T delta, T dpos, T dneg, T ev2) {
  const T eps = T(1e-30);
  if (delta > eps) {
    T num = dpos * dpos + ev2 + T(2) * delta * dpos;
    T den = dpos * dpos + T(2) * delta * delta + delta * dpos + ev2;
    return clip01(adiv(num, zmax(den, eps)));
  } else if (delta < -eps) {
    T num = dneg * dneg + ev2 + T(2) * delta * dneg;
    T den = dneg * dneg + T(2) * delta * delta + delta * dneg + ev2;
    return clip01(adiv(-num, zmin(den, -eps)));
  }
  return T(1);
}

template <typename T>
__device__ __forceinline__ T limiter_phi(int lim, T gx, T gy, T hdx, T hdy,
                                         T dpos, T dneg, T ev2) {
  if (lim == ZB_LIM_NONE) return T(1);
  T a = gx * hdx, c = gy * hdy;
  if (lim == ZB_LIM_VENKATAKRISHNAN) {
    T p = vk_cand(a, dpos, dneg, ev2);
    p = zmin(p, vk_cand(-a, dpos, dneg, ev2));
    p = zmin(p, vk_cand(c, dpos, dneg, ev2));
    p = zmin(p, vk_cand(-c, dpos, dneg, ev2));
    return clip01(p);
  }
  return phi_clipmin(a, c, dpos, dneg);
}

// ── face state and Riemann solvers ──────────────────────────────────────────
template <typename T>
struct Side {
  T b, h, qx, qy, ux, uy;
};

// Numerical flux across a face with unit normal n = sg * e_AXIS (sg = +-1).
// Outputs Fh, Fqx, Fqy and the scalar fluctuations Dm (owner / L side) and Dp
// (neighbour / R side) that multiply n.  Restates numerical_flux of the oracle:
// Rusanov (zoomy_jax/fvm/flux.py:72-82) and hydrostatic-reconstruction
// Rusanov / HLL (Audusse et al. 2004; Harten-Lax-van Leer 1983, Davis speeds).
// With an axis normal u.n = sg * u_AXIS and p n = sg * p e_AXIS exactly, so the
// terms the general form multiplies by a zero normal component are dropped.
template <typename T, int RIEMANN, int AXIS>
__device__ __forceinline__ void riemann(const Side<T>& L, const Side<T>& R, T sg, T g,
                                        T& Fh, T& Fqx, T& Fqy, T& Dm, T& Dp) {
  const T half = T(0.5);
  const T unL = sg * (AXIS == 0 ? L.ux : L.uy);
  const T unR = sg * (AXIS == 0 ? R.ux : R.uy);
  if (RIEMANN == ZB_RIEMANN_RUSANOV) {
    const T cL = asqrt(g * L.h), cR = asqrt(g * R.h);
    const T s = fmx(fabs(unL) + cL, fabs(unR) + cR);
    const T qnL = sg * (AXIS == 0 ? L.qx : L.qy);
    const T qnR = sg * (AXIS == 0 ? R.qx : R.qy);
    const T pL = sg * (half * g * (L.h * L.h)), pR = sg * (half * g * (R.h * R.h));
    T FLx = L.qx * unL, FLy = L.qy * unL, FRx = R.qx * unR, FRy = R.qy * unR;
    if (AXIS == 0) { FLx += pL; FRx += pR; } else { FLy += pL; FRy += pR; }
    const T hs = half * s;
    Fh = half * (qnL + qnR) - hs * (R.h - L.h);
    Fqx = half * (FLx + FRx) - hs * (R.qx - L.qx);
    Fqy = half * (FLy + FRy) - hs * (R.qy - L.qy);
    Dm = T(0);
    Dp = T(0);
    return;
  }
  const T bs = fmx(L.b, R.b);
  const T hLs = fmx(T(0), L.h + L.b - bs);
  const T hRs = fmx(T(0), R.h + R.b - bs);
  const T cL = asqrt(g * hLs), cR = asqrt(g * hRs);
  const T qLx = hLs * L.ux, qLy = hLs * L.uy;
  const T qRx = hRs * R.ux, qRy = hRs * R.uy;
  const T FLh = hLs * unL, FRh = hRs * unR;
  const T pL = sg * (half * g * (hLs * hLs)), pR = sg * (half * g * (hRs * hRs));
  T FLx = qLx * unL, FLy = qLy * unL, FRx = qRx * unR, FRy = qRy * unR;
  if (AXIS == 0) { FLx += pL; FRx += pR; } else { FLy += pL; FRy += pR; }
  if (RIEMANN == ZB_RIEMANN_RUSANOV_HR) {
    const T s = fmx(fabs(unL) + cL, fabs(unR) + cR);
    const T hs = half * s;
    Fh = half * (FLh + FRh) - hs * (hRs - hLs);
    Fqx = half * (FLx + FRx) - hs * (qRx - qLx);
    Fqy = half * (FLy + FRy) - hs * (qRy - qLy);
  } else {
    // Davis speeds clipped at zero: s_L = min(uL - cL, uR - cR, 0), s_R likewise
    const T sl = fmn3(unL - cL, unR - cR, T(0));
    const T sr = fmx3(unL + cL, unR + cR, T(0));
    const T den = sr - sl;
    const T inv = den > T(0) ? adiv(T(1), den) : T(0);
    const T slsr = sl * sr;
    Fh = (sr * FLh - sl * FRh + slsr * (hRs - hLs)) * inv;
    Fqx = (sr * FLx - sl * FRx + slsr * (qRx - qLx)) * inv;
    Fqy = (sr * FLy - sl * FRy + slsr * (qRy - qLy)) * inv;
  }
  Dm = half * g * (L.h * L.h - hLs * hLs);
  Dp = -(half * g * (R.h * R.h - hRs * hRs));
}

// ── one tile of one stage ───────────────────────────────────────────────────
// The body of a stage for the TX x 32 tile at (i0, j0), with the stage dt
// already decided.  Shared by the single-grid kernel (one tile per CTA) and
// the ensemble kernel (a persistent CTA walks (instance, tile) work items).
// p may live in kernel-parameter space or in global memory.
template <typename T, int TX, int ORDER, int RECON, int RIEMANN, int MODE>
__device__ __forceinline__ void stage_tile(
    Smem<T, TX>& s, double* red, const int i0, const int j0,
    const T* __restrict__ bP, const T* __restrict__ hP, const T* __restrict__ qxP,
    const T* __restrict__ qyP, const T* h0P, const T* qx0P, const T* qy0P, T* hO, T* qxO,
    T* qyO, zb_ctrl* ctrl, const int phase, const T* __restrict__ hinv_src,
    const unsigned char* __restrict__ force_o1, unsigned char* __restrict__ trouble_out,
    const SweParams<T>& p, const double dtd, const bool lead_block) {
  using S = Smem<T, TX>;
  const int tid = threadIdx.x;
  const int nx = p.nx, ny = p.ny;
  const bool per_x = p.bc[0] == ZB_BC_PERIODIC;
  const bool per_y = p.bc[2] == ZB_BC_PERIODIC;
  const T dt = T(dtd);

  // ── phase A: halo-2 load, W transform ──
  for (int e = tid; e < S::N2; e += NT) {
    const int r = e / S::R2Y, c = e - r * S::R2Y;
    int gi = i0 - 2 + r, gj = j0 - 2 + c;
    bool ix = gi >= 0 && gi < nx, iy = gj >= 0 && gj < ny;
    if (!ix && per_x && iy) { gi = (gi + nx) % nx; ix = true; }
    if (!iy && per_y && ix) { gj = (gj + ny) % ny; iy = true; }
    T vb = T(0), vh = T(0), vqx = T(0), vqy = T(0);
    if (ix && iy) {
      const size_t k = (size_t)gi * ny + gj;
      vb = bP[k]; vh = hP[k]; vqx = qxP[k]; vqy = qyP[k];
    }
    const T hinv = kp_hinv(vh, p.eps_kp);
    s.b[e] = vb;
    s.h[e] = vh;
    s.aux[e] = hinv;
    if (RECON == ZB_RECON_ETA) {
      s.w1[e] = vb + vh;
      s.w2[e] = vqx * hinv;
      s.w3[e] = vqy * hinv;
    } else {
      s.w1[e] = vh;
      s.w2[e] = vqx;
      s.w3[e] = vqy;
    }
  }
  __syncthreads();

  // ── phase B: gradients, bounds, limiter (halo-1 region) ──
  if (ORDER >= 2) {
    for (int e = tid; e < S::N1; e += NT) {
      const int r = e / S::R1Y, c = e - r * S::R1Y;
      const int gi = i0 - 1 + r, gj = j0 - 1 + c;
      if (gi < 0 || gi >= nx || gj < 0 || gj >= ny) {
#pragma unroll
        for (int v = 0; v < 4; ++v) { s.sx[v][e] = T(0); s.sy[v][e] = T(0); }
        continue;
      }
      const int e2 = (r + 1) * S::R2Y + (c + 1);
      const bool bxl = gi == 0, bxh = gi == nx - 1, byl = gj == 0, byh = gj == ny - 1;
      const bool interior = !(bxl || bxh || byl || byh);
      const int cls = (bxl ? 0 : (bxh ? 2 : 1)) * 3 + (byl ? 0 : (byh ? 2 : 1));
      const T* wv[4] = {s.b, s.w1, s.w2, s.w3};
      T phi[4], gxa[4], gya[4];
      const T ev2 = p.vk_eps2;
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const T* W = wv[v];
        const T u = W[e2];
        T gx = T(0), gy = T(0), umax = u, umin = u;
        if (interior) {
          // the unweighted 3x3 least-squares gradient of a uniform grid in
          // closed form: the normal matrix is diag(6 dx^2, 6 dy^2), so
          // g_x = (sum of the row above - sum of the row below) / (6 dx) and
          // likewise along y (u itself cancels)
          const T wmm = W[e2 - S::R2Y - 1], wm0 = W[e2 - S::R2Y], wmp = W[e2 - S::R2Y + 1];
          const T w0m = W[e2 - 1], w0p = W[e2 + 1];
          const T wpm = W[e2 + S::R2Y - 1], wp0 = W[e2 + S::R2Y], wpp = W[e2 + S::R2Y + 1];
          gx = ((wpm + wp0 + wpp) - (wmm + wm0 + wmp)) * p.inv6dx;
          gy = ((wmp + w0p + wpp) - (wmm + w0m + wpm)) * p.inv6dy;
          umax = fmx3(umax, wp0, fmx3(wm0, w0p, w0m));
          umin = fmn3(umin, wp0, fmn3(wm0, w0p, w0m));
        } else {
          // ghost values of this cell's boundary faces (BC at the cell state;
          // a wall negates the normal momentum / velocity; periodic = image)
          T gxv = u, gyv = u;
          if (bxl || bxh) {
            const int side = bxl ? 0 : 1;
            if (p.bc[side] == ZB_BC_PERIODIC) gxv = W[e2 + (bxl ? -S::R2Y : S::R2Y)];
            else if (p.bc[side] == ZB_BC_WALL && v == 2) gxv = -u;
          }
          if (byl || byh) {
            const int side = byl ? 2 : 3;
            if (p.bc[side] == ZB_BC_PERIODIC) gyv = W[e2 + (byl ? -1 : 1)];
            else if (p.bc[side] == ZB_BC_WALL && v == 3) gyv = -u;
          }
          const T* wx = p.lsq.w[cls][0];
          const T* wy = p.lsq.w[cls][1];
          int k = 0;
#pragma unroll
          for (int a = -1; a <= 1; ++a) {
#pragma unroll
            for (int bb = -1; bb <= 1; ++bb) {
              if (a == 0 && bb == 0) continue;
              const bool ok = gi + a >= 0 && gi + a < nx && gj + bb >= 0 && gj + bb < ny;
              const T d = ok ? W[e2 + a * S::R2Y + bb] - u : T(0);
              gx += wx[k] * d;
              gy += wy[k] * d;
              ++k;
            }
          }
          if (bxl || bxh) { const T d = gxv - u; gx += wx[8] * d; gy += wy[8] * d; }
          if (byl || byh) { const T d = gyv - u; gx += wx[9] * d; gy += wy[9] * d; }
          // bounds: inside face neighbours + ghost 2 u_bf - u
          if (!bxh) { umax = fmx(umax, W[e2 + S::R2Y]); umin = fmn(umin, W[e2 + S::R2Y]); }
          if (!bxl) { umax = fmx(umax, W[e2 - S::R2Y]); umin = fmn(umin, W[e2 - S::R2Y]); }
          if (!byh) { umax = fmx(umax, W[e2 + 1]); umin = fmn(umin, W[e2 + 1]); }
          if (!byl) { umax = fmx(umax, W[e2 - 1]); umin = fmn(umin, W[e2 - 1]); }
          if (bxl || bxh) { const T gg = T(2) * gxv - u; umax = fmx(umax, gg); umin = fmn(umin, gg); }
          if (byl || byh) { const T gg = T(2) * gyv - u; umax = fmx(umax, gg); umin = fmn(umin, gg); }
        }
        gxa[v] = gx;
        gya[v] = gy;
        phi[v] = limiter_phi(p.limiter, gx, gy, p.half_dx, p.half_dy,
                             umax - u, umin - u, ev2);
      }
      if (RECON == ZB_RECON_ETA) {
        if (p.eps_wet >= T(0) && s.h[e2] < p.eps_wet) {
          phi[0] = phi[1] = phi[2] = phi[3] = T(0);
        }
        phi[0] = zmin(phi[0], phi[1]);
        phi[2] = zmin(phi[2], phi[1]);
        phi[3] = zmin(phi[3], phi[1]);
      }
      if (force_o1 != nullptr && force_o1[(size_t)gi * ny + gj]) {
        phi[0] = phi[1] = phi[2] = phi[3] = T(0);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        s.sx[v][e] = phi[v] * gxa[v];
        s.sy[v][e] = phi[v] * gya[v];
      }
    }
    __syncthreads();
  }

  // ── phase C: faces ──
  // side trace of the cell at R2 index e2 / R1 index e1 at offset o along the
  // face axis (the other offset component is zero: its term is dropped)
  auto trace = [&](auto axis_tag, int e2, int e1, T o, Side<T>& sd) {
    constexpr int AX = decltype(axis_tag)::value;
    T vb = s.b[e2], w1 = s.w1[e2], w2 = s.w2[e2], w3 = s.w3[e2];
    if (ORDER >= 2) {
      if (AX == 0) {
        vb = vb + s.sx[0][e1] * o; w1 = w1 + s.sx[1][e1] * o;
        w2 = w2 + s.sx[2][e1] * o; w3 = w3 + s.sx[3][e1] * o;
      } else {
        vb = vb + s.sy[0][e1] * o; w1 = w1 + s.sy[1][e1] * o;
        w2 = w2 + s.sy[2][e1] * o; w3 = w3 + s.sy[3][e1] * o;
      }
    }
    sd.b = vb;
    if (RECON == ZB_RECON_ETA) {
      const T eta = fmx(w1, vb);
      const T hf = eta - vb;
      sd.h = hf;
      sd.ux = w2;
      sd.uy = w3;
      sd.qx = w2 * hf;
      sd.qy = w3 * hf;
    } else {
      const T hinv = s.aux[e2];
      sd.h = w1;
      sd.qx = w2;
      sd.qy = w3;
      sd.ux = w2 * hinv;
      sd.uy = w3 * hinv;
    }
  };
  using AxX = std::integral_constant<int, 0>;
  using AxY = std::integral_constant<int, 1>;
  // periodic seam: Q_R is the partner cell's (unreconstructed) state; its
  // velocity is the partner's own W row on the eta path and q times the
  // OWNER's hinv on the conservative path (the flux pass hands the inner
  // cell's aux to both sides of a boundary face, solver_jax.py:827-866)
  auto partner = [&](int e2img, T hinv_owner, Side<T>& sd) {
    sd.b = s.b[e2img];
    sd.h = s.h[e2img];
    if (RECON == ZB_RECON_ETA) {
      sd.ux = s.w2[e2img];
      sd.uy = s.w3[e2img];
      sd.qx = sd.ux * sd.h;   // not read by the hydrostatic-reconstruction fluxes
      sd.qy = sd.uy * sd.h;
    } else {
      sd.qx = s.w2[e2img];
      sd.qy = s.w3[e2img];
      sd.ux = sd.qx * hinv_owner;
      sd.uy = sd.qy * hinv_owner;
    }
  };
  const T g = p.g;
  const T half = T(0.5);
  // x-faces
  for (int e = tid; e < S::NFX; e += NT) {
    const int fi = e / TY, fj = e - fi * TY;
    const int gi = i0 + fi, gj = j0 + fj;
    if (gj >= ny || gi > nx) continue;
    const int e2L = (fi + 1) * S::R2Y + (fj + 2), e2R = e2L + S::R2Y;
    const int e1L = fi * S::R1Y + (fj + 1), e1R = e1L + S::R1Y;
    Side<T> A, B;
    T Fh, Fx, Fy, Dm, Dp;
    if (gi == 0 || gi == nx) {
      const bool lo = gi == 0;
      const int e2o = lo ? e2R : e2L, e1o = lo ? e1R : e1L;
      const T sg = lo ? T(-1) : T(1);
      trace(AxX(), e2o, e1o, sg * p.half_dx, A);
      const int kind = p.bc[lo ? 0 : 1];
      if (kind == ZB_BC_PERIODIC) {
        partner(lo ? e2L : e2R, s.aux[e2o], B);
      } else {
        B = A;
        if (kind == ZB_BC_WALL) {   // q - 2 (q.n) n with n = (sg, 0): q_x -> -q_x
          B.qx = -A.qx;
          B.ux = -A.ux;
        }
      }
      riemann<T, RIEMANN, 0>(A, B, sg, g, Fh, Fx, Fy, Dm, Dp);
      T ces = T(0);
      if (ORDER >= 2) ces = half * g * (s.h[e2o] + A.h) * (A.b - s.b[e2o]);
      const T own_n = Fx + Dm * sg + ces * sg;
      if (lo) {
        s.fxh[e] = -Fh; s.fxt[e] = -Fy; s.fxr[e] = own_n; s.fxl[e] = T(0);
      } else {
        s.fxh[e] = Fh; s.fxt[e] = Fy; s.fxl[e] = own_n; s.fxr[e] = T(0);
      }
    } else {
      trace(AxX(), e2L, e1L, p.half_dx, A);
      trace(AxX(), e2R, e1R, -p.half_dx, B);
      riemann<T, RIEMANN, 0>(A, B, T(1), g, Fh, Fx, Fy, Dm, Dp);
      T cesA = T(0), cesB = T(0);
      if (ORDER >= 2) {
        cesA = half * g * (s.h[e2L] + A.h) * (A.b - s.b[e2L]);
        cesB = -(half * g * (s.h[e2R] + B.h) * (B.b - s.b[e2R]));
      }
      s.fxh[e] = Fh;
      s.fxt[e] = Fy;
      s.fxl[e] = Fx + Dm + cesA;
      s.fxr[e] = -Fx + Dp + cesB;
    }
  }
  // y-faces
  for (int e = tid; e < S::NFY; e += NT) {
    const int fi = e / (TY + 1), fj = e - fi * (TY + 1);
    const int gi = i0 + fi, gj = j0 + fj;
    if (gi >= nx || gj > ny) continue;
    const int e2L = (fi + 2) * S::R2Y + (fj + 1), e2R = e2L + 1;
    const int e1L = (fi + 1) * S::R1Y + fj, e1R = e1L + 1;
    Side<T> A, B;
    T Fh, Fx, Fy, Dm, Dp;
    if (gj == 0 || gj == ny) {
      const bool lo = gj == 0;
      const int e2o = lo ? e2R : e2L, e1o = lo ? e1R : e1L;
      const T sg = lo ? T(-1) : T(1);
      trace(AxY(), e2o, e1o, sg * p.half_dy, A);
      const int kind = p.bc[lo ? 2 : 3];
      if (kind == ZB_BC_PERIODIC) {
        partner(lo ? e2L : e2R, s.aux[e2o], B);
      } else {
        B = A;
        if (kind == ZB_BC_WALL) {   // n = (0, sg): q_y -> -q_y
          B.qy = -A.qy;
          B.uy = -A.uy;
        }
      }
      riemann<T, RIEMANN, 1>(A, B, sg, g, Fh, Fx, Fy, Dm, Dp);
      T ces = T(0);
      if (ORDER >= 2) ces = half * g * (s.h[e2o] + A.h) * (A.b - s.b[e2o]);
      const T own_n = Fy + Dm * sg + ces * sg;
      if (lo) {
        s.fyh[e] = -Fh; s.fyt[e] = -Fx; s.fyr[e] = own_n; s.fyl[e] = T(0);
      } else {
        s.fyh[e] = Fh; s.fyt[e] = Fx; s.fyl[e] = own_n; s.fyr[e] = T(0);
      }
    } else {
      trace(AxY(), e2L, e1L, p.half_dy, A);
      trace(AxY(), e2R, e1R, -p.half_dy, B);
      riemann<T, RIEMANN, 1>(A, B, T(1), g, Fh, Fx, Fy, Dm, Dp);
      T cesA = T(0), cesB = T(0);
      if (ORDER >= 2) {
        cesA = half * g * (s.h[e2L] + A.h) * (A.b - s.b[e2L]);
        cesB = -(half * g * (s.h[e2R] + B.h) * (B.b - s.b[e2R]));
      }
      s.fyh[e] = Fh;
      s.fyt[e] = Fx;
      s.fyl[e] = Fy + Dm + cesA;
      s.fyr[e] = -Fy + Dp + cesB;
    }
  }
  __syncthreads();

  // ── phase D: divergence, stage update, epilogue ──
  double amax_loc = 0.0;
  bool bad = false;
  for (int e = tid; e < TX * TY; e += NT) {
    const int ti = e / TY, tj = e - ti * TY;
    const int gi = i0 + ti, gj = j0 + tj;
    if (gi >= nx || gj >= ny) continue;
    // cells of the interior strip kernel's region are its to write
    if (gi >= p.fast_i0 && gi < p.fast_i1 && gj >= p.fast_j0 && gj < p.fast_j1) continue;
    const int fl = ti * TY + tj, fr = fl + TY;
    const int fb = ti * (TY + 1) + tj, ft = fb + 1;
    const T kx = p.kx, ky = p.ky;
    const T dh = -(kx * (s.fxh[fr] - s.fxh[fl]) + ky * (s.fyh[ft] - s.fyh[fb]));
    const T dqx = -(kx * (s.fxl[fr] + s.fxr[fl]) + ky * (s.fyt[ft] - s.fyt[fb]));
    const T dqy = -(kx * (s.fxt[fr] - s.fxt[fl]) + ky * (s.fyl[ft] + s.fyr[fb]));
    const int e2 = (ti + 2) * S::R2Y + (tj + 2);
    const T hk = s.h[e2];
    T qxk, qyk;
    if (RECON == ZB_RECON_ETA) {
      const size_t k = (size_t)gi * ny + gj;
      qxk = qxP[k];
      qyk = qyP[k];
    } else {
      qxk = s.w2[e2];
      qyk = s.w3[e2];
    }
    T hn, qxn, qyn;
    const size_t k = (size_t)gi * ny + gj;
    if (MODE == MODE_STEP1) {
      hn = hk + dt * dh;
      qxn = qxk + dt * dqx;
      qyn = qyk + dt * dqy;
    } else if (MODE == MODE_STEP2) {
      const T h2 = hk + dt * dh, qx2 = qxk + dt * dqx, qy2 = qyk + dt * dqy;
      const T h0 = h0P[k], qx0 = qx0P[k], qy0 = qy0P[k];
      hn = half * (h0 + h2);
      qxn = half * (qx0 + qx2);
      qyn = half * (qy0 + qy2);
    } else if (MODE == MODE_EULER) {
      hn = hk + dt * dh;
      qxn = qxk + dt * dqx;
      qyn = qyk + dt * dqy;
    } else {
      const T a = T(p.alpha), bt = T(p.beta);
      T sqx = dqx, sqy = dqy;
      if (hinv_src != nullptr && p.manning_n != T(0)) {
        // solver2 adds the source to the stage residual at Qk with the step's
        // aux (solver2/blocks.py:241-287, march.py:120-124)
        const T hi = hinv_src[k];
        const T qn = asqrt(qxk * qxk + qyk * qyk);
        const T kf = (-p.g) * (p.manning_n * p.manning_n) * qn * (hi * hi) * cbrt(hi);
        sqx = dqx + qxk * kf;
        sqy = dqy + qyk * kf;
      }
      const T h2 = hk + bt * dt * dh, qx2 = qxk + bt * dt * sqx, qy2 = qyk + bt * dt * sqy;
      if (p.alpha != 0.0) {
        const T h0 = h0P[k], qx0 = qx0P[k], qy0 = qy0P[k];
        hn = a * h0 + (T(1) - a) * h2;
        qxn = a * qx0 + (T(1) - a) * qx2;
        qyn = a * qy0 + (T(1) - a) * qy2;
      } else {
        hn = h2; qxn = qx2; qyn = qy2;
      }
    }
    if ((MODE == MODE_STEP2 || MODE == MODE_EULER) && p.manning_n != T(0)) {
      // source as RK1 after the hyperbolic step with the step's input aux
      // (zoomy_jax/fvm/solver_jax.py:1129; ode.py:14-18)
      const T h0 = (MODE == MODE_STEP2) ? h0P[k] : hk;
      const T hi0 = kp_hinv(h0, p.eps_kp);
      const T qn = asqrt(qxn * qxn + qyn * qyn);
      const T kf = (-p.g) * (p.manning_n * p.manning_n) * qn * (hi0 * hi0) * cbrt(hi0);
      if (p.implicit_source) {
        const T den = T(1) + dt * (-kf);
        qxn = qxn / den;
        qyn = qyn / den;
      } else {
        qxn = qxn + dt * (qxn * kf);
        qyn = qyn + dt * (qyn * kf);
      }
    }
    hO[k] = hn;
    qxO[k] = qxn;
    qyO[k] = qyn;
    const bool tr = (hn < T(0)) || !isfinite(hn) || !isfinite(qxn) || !isfinite(qyn) ||
                    !isfinite(s.b[e2]);
    bad = bad || tr;
    if (trouble_out != nullptr) trouble_out[k] = tr ? 1 : 0;
    if (MODE == MODE_STEP2 || MODE == MODE_EULER) {
      const T hi = kp_hinv(hn, p.eps_kp);
      const T c = asqrt(g * fmx(hn, T(0)));
      const T lx = fabs(qxn * hi) + c, ly = fabs(qyn * hi) + c;
      amax_loc = nmax(amax_loc, (double)nmax(lx, ly));
    }
  }
  const unsigned anybad = __syncthreads_or(bad ? 1 : 0);
  if (anybad && tid == 0) atomicOr(&ctrl->status, (unsigned)ZB_ST_TROUBLED);
  if (MODE == MODE_STEP2 || MODE == MODE_EULER) {
    const double m = block_max_double(amax_loc, red);
    if (tid == 0) {
      atomic_max_pos_double(&ctrl->amax[(phase + 1) % 3], m);
      if (lead_block) atomicAdd(&ctrl->steps, 1u);
    }
  }
}

// ── the fused stage kernel (one tile per CTA) ───────────────────────────────
template <typename T, int TX, int ORDER, int RECON, int RIEMANN, int MODE>
__global__ void __launch_bounds__(NT)
swe2d_stage_kernel(const T* __restrict__ bP, const T* __restrict__ hP,
                   const T* __restrict__ qxP, const T* __restrict__ qyP,
                   const T* h0P, const T* qx0P, const T* qy0P,
                   T* hO, T* qxO, T* qyO, zb_ctrl* ctrl, int phase,
                   const T* __restrict__ hinv_src,
                   const unsigned char* __restrict__ force_o1,
                   unsigned char* __restrict__ trouble_out,
                   const SweParams<T> p) {
  using S = Smem<T, TX>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& s = *reinterpret_cast<S*>(smem_raw);
  __shared__ double red[NT / 32];

  const int tid = threadIdx.x;
  int i0 = blockIdx.y * TX, j0 = blockIdx.x * TY;
  if (p.fast_i1 > p.fast_i0) {
    // frame launch (1-D grid): enumerate only the tiles that hold cells outside
    // the strip kernel's region -- whole tile rows above and below it, then
    // the tile columns left and right of it for the rows in between
    const int ntc = (p.ny + TY - 1) / TY, ntr = (p.nx + TX - 1) / TX;
    // (bands never overlap: a region narrower than a tile leaves tcb = tca)
    const int tra = (p.fast_i0 + TX - 1) / TX, trb = max(tra, p.fast_i1 / TX);
    const int tca = (p.fast_j0 + TY - 1) / TY, tcb = max(tca, p.fast_j1 / TY);
    const int nside = tca + (ntc - tcb);
    int b = blockIdx.x;
    if (b < tra * ntc) {
      i0 = (b / ntc) * TX; j0 = (b % ntc) * TY;
    } else if ((b -= tra * ntc) < (ntr - trb) * ntc) {
      i0 = (trb + b / ntc) * TX; j0 = (b % ntc) * TY;
    } else {
      b -= (ntr - trb) * ntc;
      const int tr = tra + b / nside, k = b % nside;
      i0 = tr * TX;
      j0 = (k < tca ? k : tcb + (k - tca)) * TY;
    }
  }

  // dt of this step
  double dtd;
  if (MODE == MODE_STAGE) {
    dtd = p.dt_stage >= 0.0 ? p.dt_stage : ctrl->dt;
  } else {
    const int ph = phase;
    const int nph = (ph + 1) % 3, nnph = (ph + 2) % 3;
    const double t = ctrl->t[ph];
    dtd = dt_from_amax(ctrl->amax[ph], t, p.cfl2r, p.den_fac, p.dt_max, p.t_end);
    const bool ok = isfinite(dtd) && dtd > 0.0;
    const bool lead = blockIdx.x == 0 && blockIdx.y == 0 && tid == 0;
    if ((MODE == MODE_STEP1 || MODE == MODE_EULER) && lead) {
      if (!ok && t < p.t_end) atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
      ctrl->dt = ok ? dtd : 0.0;
      ctrl->t[nph] = ok ? t + dtd : t;
      ctrl->amax[nnph] = 0.0;
      ctrl->troubled = 0u;
    }
    if (!ok) {
      // no-op step (t_end reached or dt invalid): the state is unchanged, so
      // the next slot carries this slot's wave-speed maximum forward
      if ((MODE == MODE_STEP2 || MODE == MODE_EULER) && lead) ctrl->amax[nph] = ctrl->amax[ph];
      if (MODE == MODE_EULER) {
        // the Euler path writes the workspace that is copied back: keep it equal
        const int nx_ = p.nx, ny_ = p.ny;
        for (int e = tid; e < TX * TY; e += NT) {
          const int gi = i0 + e / TY, gj = j0 + e % TY;
          if (gi < nx_ && gj < ny_) {
            const size_t k = (size_t)gi * ny_ + gj;
            hO[k] = hP[k]; qxO[k] = qxP[k]; qyO[k] = qyP[k];
          }
        }
      }
      return;
    }
  }
  // a tile wholly inside the strip kernel's region has nothing to write (the
  // lead block sits at the corner, outside the region)
  if (i0 >= p.fast_i0 && i0 + TX <= p.fast_i1 && j0 >= p.fast_j0 && j0 + TY <= p.fast_j1) return;
  stage_tile<T, TX, ORDER, RECON, RIEMANN, MODE>(
      s, red, i0, j0, bP, hP, qxP, qyP, h0P, qx0P, qy0P, hO, qxO, qyO, ctrl, phase, hinv_src,
      force_o1, trouble_out, p, dtd, blockIdx.x == 0 && blockIdx.y == 0);
}


// ── the strip kernel ───────────────────────────────────────────────────────
// The stage arithmetic of stage_tile organised for registers instead of
// shared memory: one warp owns a strip of 32 contiguous columns (28 outputs
// plus two halo columns on each side) and marches down its rows.  Each lane
// keeps a sliding window of three rows of W, the limited slopes of two rows
// and the last x-face's fluxes in registers; the column neighbours come from
// warp shuffles.  Every face is still evaluated once.  Interior items (every
// cell two cells from every boundary) take the interior body, which for
// float64 evaluates stage_tile's float expressions (the same bits); items
// that reach the boundary rows take the EDGE body, items whose rows are inside
// but whose lanes reach a boundary column the column-EDGE body (strip_item
// below).
constexpr int SX = 64;          // output rows per work item
constexpr int SW = 28;          // output columns per strip
constexpr int STRIP_NT = 128;   // four independent warps per CTA
constexpr int SXC_MAX = 32;     // output rows of the longest column-EDGE item

template <typename T>
struct RowW {
  T b, w1, w2, w3, h, hinv;
  __device__ T w(int v) const { return v == 0 ? b : (v == 1 ? w1 : (v == 2 ? w2 : w3)); }
};

template <typename T, int RECON>
__device__ __forceinline__ void strip_trace(const RowW<T>& c, const T* sl, T o, Side<T>& sd) {
  const T vb = c.b + sl[0] * o, w1 = c.w1 + sl[1] * o;
  const T w2 = c.w2 + sl[2] * o, w3 = c.w3 + sl[3] * o;
  sd.b = vb;
  if (RECON == ZB_RECON_ETA) {
    const T eta = fmx(w1, vb);
    const T hf = eta - vb;
    sd.h = hf;
    sd.ux = w2;
    sd.uy = w3;
    sd.qx = w2 * hf;
    sd.qy = w3 * hf;
  } else {
    sd.h = w1;
    sd.qx = w2;
    sd.qy = w3;
    sd.ux = w2 * c.hinv;
    sd.uy = w3 * c.hinv;
  }
}

template <typename T>
__device__ __forceinline__ T shd(T v) { return __shfl_down_sync(0xffffffffu, v, 1); }
template <typename T>
__device__ __forceinline__ T shu(T v) { return __shfl_up_sync(0xffffffffu, v, 1); }

// float2 arithmetic on the sm_100 paired-FP32 instructions (one issue slot for
// two lanes of the same operation)
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {   // a - b, one rounding
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// The x-face (rows r-2 | r-1) and the y-face (row r-2, this lane | next lane)
// of an interior strip row evaluated together as the two lanes of float2
// arithmetic: eta traces, the Audusse hydrostatic reconstruction, HLL with
// Davis speeds, the fluctuations and the cell-edge bed terms of riemann() and
// strip_trace() for ZB_RECON_ETA / ZB_RIEMANN_HLL_HR in float32.  Lane x is
// the x-face (normal velocity u, transverse v), lane y the y-face (normal v,
// transverse u).  Square roots, divisions and min / max stay per lane.
// Outputs as the scalar path names them: x-face Fh, Fy, fxl_n, fxr_n; y-face
// Gh, Gx, fyl_t, fyr_own.
// The next lane's row r-2 (the y-face's upper side): W, h and the y-slopes.
struct NextRow {
  float b, w1, w2, w3, h, s4, s5, s6, s7;
};
__device__ __forceinline__ NextRow next_row(const RowW<float>& R0, const float* slA) {
  NextRow n;
  n.b = shd(R0.b); n.w1 = shd(R0.w1); n.w2 = shd(R0.w2); n.w3 = shd(R0.w3); n.h = shd(R0.h);
  n.s4 = shd(slA[4]); n.s5 = shd(slA[5]); n.s6 = shd(slA[6]); n.s7 = shd(slA[7]);
  return n;
}

__device__ __forceinline__ void faces_pair(const RowW<float>& R0, const RowW<float>& R1,
                                           const float* slA, const float* slB,
                                           const NextRow& nx_, const SweParams<float>& p,
                                           float& Fh, float& Fy, float& fxl_n, float& fxr_n,
                                           float& Gh, float& Gx, float& fyl_t, float& fyr_own) {
  const float g = p.g, hg = 0.5f * g;
  const float nb_b = nx_.b, nb_w1 = nx_.w1, nb_w2 = nx_.w2, nb_w3 = nx_.w3, nb_h = nx_.h;
  const float sn4 = nx_.s4, sn5 = nx_.s5, sn6 = nx_.s6, sn7 = nx_.s7;
  const float2 o1 = f2(p.half_dx, p.half_dy), o2 = f2(-p.half_dx, -p.half_dy);
  // side 1: row r-2 towards +x (x-face) and towards +y (y-face)
  const float2 b1 = fma2(f2(slA[0], slA[4]), o1, f2(R0.b, R0.b));
  const float2 e1 = fma2(f2(slA[1], slA[5]), o1, f2(R0.w1, R0.w1));
  const float2 un1 = fma2(f2(slA[2], slA[7]), o1, f2(R0.w2, R0.w3));
  const float2 ut1 = fma2(f2(slA[3], slA[6]), o1, f2(R0.w3, R0.w2));
  const float2 h1 = sub2(f2(fmaxf(e1.x, b1.x), fmaxf(e1.y, b1.y)), b1);   // Audusse clip
  // side 2: row r-1 towards -x and the next lane's row r-2 towards -y
  const float2 b2 = fma2(f2(slB[0], sn4), o2, f2(R1.b, nb_b));
  const float2 e2 = fma2(f2(slB[1], sn5), o2, f2(R1.w1, nb_w1));
  const float2 un2 = fma2(f2(slB[2], sn7), o2, f2(R1.w2, nb_w3));
  const float2 ut2 = fma2(f2(slB[3], sn6), o2, f2(R1.w3, nb_w2));
  const float2 h2 = sub2(f2(fmaxf(e2.x, b2.x), fmaxf(e2.y, b2.y)), b2);
  // hydrostatic reconstruction
  const float2 bs = f2(fmaxf(b1.x, b2.x), fmaxf(b1.y, b2.y));
  const float2 t1 = sub2(add2(h1, b1), bs), t2 = sub2(add2(h2, b2), bs);
  const float2 hL = f2(fmaxf(0.f, t1.x), fmaxf(0.f, t1.y));
  const float2 hR = f2(fmaxf(0.f, t2.x), fmaxf(0.f, t2.y));
  const float2 gg = f2(g, g), hg2 = f2(hg, hg), m1 = f2(-1.f, -1.f);
  const float2 ghL = mul2(gg, hL), ghR = mul2(gg, hR);
  const float2 cL = f2(sqrtf(ghL.x), sqrtf(ghL.y)), cR = f2(sqrtf(ghR.x), sqrtf(ghR.y));
  const float2 FLh = mul2(hL, un1), FRh = mul2(hR, un2);      // normal discharges
  const float2 qLt = mul2(hL, ut1), qRt = mul2(hR, ut2);      // transverse discharges
  const float2 FLn = fma2(FLh, un1, mul2(hg2, mul2(hL, hL)));
  const float2 FRn = fma2(FRh, un2, mul2(hg2, mul2(hR, hR)));
  const float2 FLt = mul2(qLt, un1), FRt = mul2(qRt, un2);
  // Davis speeds clipped at zero and the HLL combination
  const float2 sL1 = sub2(un1, cL), sL2 = sub2(un2, cR), sR1 = add2(un1, cL), sR2 = add2(un2, cR);
  const float2 sl = f2(fmn3(sL1.x, sL2.x, 0.f), fmn3(sL1.y, sL2.y, 0.f));
  const float2 sr = f2(fmx3(sR1.x, sR2.x, 0.f), fmx3(sR1.y, sR2.y, 0.f));
  const float2 den = sub2(sr, sl);
  const float2 inv = f2(den.x > 0.f ? __fdividef(1.f, den.x) : 0.f,
                        den.y > 0.f ? __fdividef(1.f, den.y) : 0.f);
  const float2 slsr = mul2(sl, sr), nsl = mul2(sl, m1);
  auto hll = [&](float2 FL, float2 FR, float2 d) {
    return mul2(fma2(slsr, d, fma2(nsl, FR, mul2(sr, FL))), inv);
  };
  const float2 Fh2 = hll(FLh, FRh, sub2(hR, hL));
  const float2 Fn2 = hll(FLn, FRn, sub2(FRh, FLh));
  const float2 Ft2 = hll(FLt, FRt, sub2(qRt, qLt));
  // fluctuations of the reconstruction and the cell-edge bed terms
  const float2 Dm2 = mul2(hg2, fma2(mul2(hL, m1), hL, mul2(h1, h1)));
  const float2 Dp2 = mul2(f2(-hg, -hg), fma2(mul2(hR, m1), hR, mul2(h2, h2)));
  const float2 ces1 = mul2(mul2(hg2, add2(f2(R0.h, R0.h), h1)), sub2(b1, f2(R0.b, R0.b)));
  const float2 ces2 = mul2(mul2(f2(-hg, -hg), add2(f2(R1.h, nb_h), h2)), sub2(b2, f2(R1.b, nb_b)));
  const float2 fl = add2(add2(Fn2, Dm2), ces1);
  const float2 fr = add2(sub2(Dp2, Fn2), ces2);
  Fh = Fh2.x; Fy = Ft2.x; fxl_n = fl.x; fxr_n = fr.x;
  Gh = Fh2.y; Gx = Ft2.y; fyl_t = fl.y; fyr_own = fr.y;
}

// Column-EDGE pre-pass for one row: the boundary column's cell (m, c), c = 0
// (low side) or ny - 1, m two cells or more from the x boundaries.  out[0..8):
// its limited slopes [sx0..3, sy0..3] (the EDGE body's side-class closed form,
// limiter, dry demotion and ties); out[8..12): Gh, Gx, fyl_t, fyr_own of its
// boundary y-face (the owner's trace against its ghost with normal sign sgy),
// as the EDGE body leaves them on the lane that evaluates that face (cj = -1
// for the low side, cj = ny - 1 for the high side).
template <typename T, int RECON, int RIEMANN>
__device__ __forceinline__ void bcol_row(const T* __restrict__ bP, const T* __restrict__ hP,
                                         const T* __restrict__ qxP, const T* __restrict__ qyP,
                                         const SweParams<T>& p, int m, int c, T* out) {
  const int ny = p.ny;
  const bool lo = c == 0;
  const int ci = lo ? 1 : ny - 2;
  RowW<T> Wc[3], Wi[3];   // rows m - 1, m, m + 1 of column c and of its inner neighbour ci
#pragma unroll
  for (int a = 0; a < 3; ++a) {
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      const size_t k = (size_t)(m - 1 + a) * ny + (s ? ci : c);
      const T vb = bP[k], vh = hP[k], vqx = qxP[k], vqy = qyP[k];
      RowW<T>& w = s ? Wi[a] : Wc[a];
      const T hinv = kp_hinv(vh, p.eps_kp);
      w.b = vb;
      w.h = vh;
      w.hinv = hinv;
      if (RECON == ZB_RECON_ETA) {
        w.w1 = vb + vh; w.w2 = vqx * hinv; w.w3 = vqy * hinv;
      } else {
        w.w1 = vh; w.w2 = vqx; w.w3 = vqy;
      }
    }
  }
  const bool wall = p.bc[lo ? 2 : 3] == ZB_BC_WALL;
  T gx[4], gy[4], phi[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const T u = Wc[1].w(v);
    const T gyv = (wall && v == 3) ? -u : u;
    const T n0 = Wi[0].w(v), n1 = Wi[1].w(v), n2 = Wi[2].w(v);
    gx[v] = ((Wc[2].w(v) + n2) - (Wc[0].w(v) + n0)) * p.inv4dx;
    const T sn = (n0 + n1) + n2;
    gy[v] = (lo ? (sn - gyv) - T(2) * u : (gyv + T(2) * u) - sn) * p.inv4dy;
    const T gg = T(2) * gyv - u;
    const T umax = fmx(fmx(fmx(fmx(u, Wc[2].w(v)), Wc[0].w(v)), n1), gg);
    const T umin = fmn(fmn(fmn(fmn(u, Wc[2].w(v)), Wc[0].w(v)), n1), gg);
    phi[v] = limiter_phi(p.limiter, gx[v], gy[v], p.half_dx, p.half_dy, umax - u, umin - u,
                         p.vk_eps2);
  }
  if (RECON == ZB_RECON_ETA) {
    if (p.eps_wet >= T(0) && Wc[1].h < p.eps_wet) phi[0] = phi[1] = phi[2] = phi[3] = T(0);
    phi[0] = zmin(phi[0], phi[1]);
    phi[2] = zmin(phi[2], phi[1]);
    phi[3] = zmin(phi[3], phi[1]);
  }
  T sy[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    out[v] = phi[v] * gx[v];
    out[4 + v] = sy[v] = phi[v] * gy[v];
  }
  Side<T> O;
  strip_trace<T, RECON>(Wc[1], sy, lo ? -p.half_dy : p.half_dy, O);
  Side<T> G = O;
  if (wall) {
    G.qy = -O.qy;
    G.uy = -O.uy;
  }
  const T sgy = lo ? T(-1) : T(1);
  T Gh, Gx, Gy, Em, Ep;
  riemann<T, RIEMANN, 1>(O, G, sgy, p.g, Gh, Gx, Gy, Em, Ep);
  // the owner's cell-edge bed term: cesC of the high side, -cesD of the low
  const T ces = T(0.5) * p.g * (Wc[1].h + O.h) * (O.b - Wc[1].b);
  const T own_n = Gy + Em * sgy + ces * sgy;
  out[8] = lo ? -Gh : Gh;
  out[9] = lo ? -Gx : Gx;
  out[10] = lo ? T(0) : own_n;
  out[11] = lo ? own_n : T(0);
}

// One warp's work item: strip `strip` (28 output columns) over the output rows
// [r0, r1) of the strip region p.fast_*.  EK selects the body:
//   0  interior: every lane's cell two cells or more from every boundary;
//   1  EDGE (full-coverage mode, wall / extrapolation sides only): rows and
//      columns outside the grid are ghosts that load nothing, boundary cells
//      take the least-squares class weights and the ghost values of their
//      sides, and the faces on the boundary take the side's ghost state -- the
//      expressions of stage_tile's boundary branches;
//   2  column EDGE: the rows [r0 - 2, r1 + 2) lie inside the grid (r0 >= 2,
//      r1 <= nx - 2) but the strip's lanes reach a boundary column: the
//      interior body with guarded column loads; the boundary column's slopes
//      and its boundary y-face by the EDGE expressions, recomputed on the
//      lanes that hold them, row by row;
//   3  column EDGE as 2, but for the paired float32 body the boundary
//      columns' slopes and y-faces of every row of the item come from a
//      pre-pass that evaluates them one row per lane (bcol_row) into shared
//      memory: for long items (the ensemble's), whose march it frees of the
//      one-lane row-by-row work; a short item's pre-pass is latency it cannot
//      hide (measured on the single grid's 8-row items: 0.189 -> 0.211 ms per
//      step, where the 32-row ensemble items gain 2.10 -> 1.92 ms).
// `lead` (one item of the grid in full-coverage mode, where no tile kernel
// runs) keeps the control block.
template <typename T, int RECON, int RIEMANN, int MODE, int EK, bool BEDT = false>
__device__ __forceinline__ void strip_item(const T* __restrict__ bP, const T* __restrict__ hP,
                                           const T* __restrict__ qxP, const T* __restrict__ qyP,
                                           const T* __restrict__ h0P,
                                           const T* __restrict__ qx0P,
                                           const T* __restrict__ qy0P, T* __restrict__ hO,
                                           T* __restrict__ qxO, T* __restrict__ qyO,
                                           zb_ctrl* ctrl, int phase, const SweParams<T>& p,
                                           const int strip, const int r0, const int r1,
                                           const bool lead) {
  constexpr bool EDGE = EK == 1;   // row and column guards
  constexpr bool CG = EK != 0;     // column guards
  const int lane = threadIdx.x & 31;
  const int nx = p.nx, ny = p.ny;
  const int cj = p.fast_j0 - 2 + strip * SW + lane;
  const bool colv = !CG || (cj >= 0 && cj < ny);
  const double t = ctrl->t[phase];
  const double dtd = dt_from_amax(ctrl->amax[phase], t, p.cfl2r, p.den_fac, p.dt_max, p.t_end);
  const bool ok = isfinite(dtd) && dtd > 0.0;
  if (lead && lane == 0) {
    // the duties of the tile kernel's lead block (swe2d_stage_kernel)
    const int nph = (phase + 1) % 3, nnph = (phase + 2) % 3;
    if (MODE == MODE_STEP1) {
      if (!ok && t < p.t_end) atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
      ctrl->dt = ok ? dtd : 0.0;
      ctrl->t[nph] = ok ? t + dtd : t;
      ctrl->amax[nnph] = 0.0;
      ctrl->troubled = 0u;
    } else if (!ok) {
      ctrl->amax[nph] = ctrl->amax[phase];
    } else {
      atomicAdd(&ctrl->steps, 1u);
    }
  }
  if (!ok) return;                      // no-op step (t_end reached or dt invalid)
  const T dt = T(dtd);
  const T g = p.g, half = T(0.5);
  const bool out_lane = lane >= 2 && lane < 2 + SW && (!CG || cj < ny);
  // float32 interior rows of the eta / HLL-HR scheme evaluate their two faces
  // as paired float32 arithmetic (faces_pair)
  constexpr bool PAIR = std::is_same<T, float>::value && RECON == ZB_RECON_ETA &&
                        RIEMANN == ZB_RIEMANN_HLL_HR && !EDGE;
  // column-EDGE with the paired body: the boundary columns' rows come from
  // the pre-pass, slots [side][m - (r0 - 1)][12] of this warp (side 0: column
  // 0, side 1: column ny - 1; rows r0 - 1 .. r1)
  constexpr bool PRE = EK == 3 && PAIR;
  // BEDT: interior items of the eta / HLL-HR scheme read b's gradient and
  // limiter value from the planes swe2d_bed_kernel prepared (b never
  // changes) instead of evaluating them; the planes are laid out like the
  // state's
  constexpr bool BED = BEDT && EK == 0 && RECON == ZB_RECON_ETA && RIEMANN == ZB_RIEMANN_HLL_HR;
  const T* __restrict__ bedP = p.bed;
  const size_t bed_plane = (size_t)nx * ny;
  constexpr int PROWS = SXC_MAX + 2;
  T* bs = nullptr;
  if constexpr (PRE) {
    __shared__ T bsh[STRIP_NT / 32][2 * PROWS * 12];
    bs = bsh[threadIdx.x >> 5];
    const int cj0 = p.fast_j0 - 2 + strip * SW;
    const int nrows = r1 - r0 + 2;   // <= SXC_MAX + 2 (full_items)
    __syncwarp();                      // the warp's previous item is done with the slots
    for (int side = 0; side < 2; ++side) {
      const int c = side ? ny - 1 : 0;
      if (!(cj0 <= c && c <= cj0 + 31)) continue;   // warp-uniform
      for (int mm = lane; mm < nrows; mm += 32)
        bcol_row<T, RECON, RIEMANN>(bP, hP, qxP, qyP, p, r0 - 1 + mm, c,
                                    bs + (side * PROWS + mm) * 12);
    }
    __syncwarp();
  }

  RowW<T> R0, R1, R2;                 // rows r-2, r-1, r
  T Sx0[4], Sx1[4], Sx2[4];           // (W(j-1) + W(j)) + W(j+1) of those rows
  T Wm1[4], Wp1[4], Wm2[4], Wp2[4];   // W(j-1), W(j+1) of rows r-1 and r
  T slA[8], slB[8];                   // [sx0..3, sy0..3] of rows r-2 and r-1
  T fxh_p = T(0), fxt_p = T(0), fxr_p = T(0);
  T amax_loc = T(0);   // reduced in T; float -> double is exact and monotone
  bool bad = false;
  const int nsteps = (r1 - r0) + 4;
  // row r + 1 is fetched while row r is processed
  T nbv = T(0), nhv = T(0), nqxv = T(0), nqyv = T(0);
  T nbgx = T(0), nbgy = T(0), nbphi = T(0);   // BED: the next slope row's bed values
  if (!CG || (colv && (!EDGE || r0 - 2 >= 0))) {
    const size_t k = (size_t)(r0 - 2) * ny + cj;
    nbv = bP[k]; nhv = hP[k]; nqxv = qxP[k]; nqyv = qyP[k];
  }
  for (int s = 0; s < nsteps; ++s) {
    const int r = r0 - 2 + s;
    // the update of row r - 2 at the end of this iteration reads these: issue
    // the loads now so their latency overlaps the slope and face work
    const int ro = r - 2;
    const bool upd = s >= 4 && out_lane && ro >= r0 && ro < r1;
    T qxk = T(0), qyk = T(0), h0 = T(0), qx0 = T(0), qy0 = T(0);
    if (upd) {
      const size_t k = (size_t)ro * ny + cj;
      if (RECON == ZB_RECON_ETA) { qxk = qxP[k]; qyk = qyP[k]; }
      if (MODE == MODE_STEP2) { h0 = h0P[k]; qx0 = qx0P[k]; qy0 = qy0P[k]; }
    }
    // the bed slopes of row r - 1 (the slope block below), fetched in the
    // previous iteration; fetch row r's for the next one
    const T bgx = nbgx, bgy = nbgy, bphi = nbphi;
    if (BED && s >= 1 && r <= r1) {
      const size_t k = (size_t)r * ny + cj;   // BED: EK == 0, no guards
      nbgx = __ldg(bedP + k);
      nbgy = __ldg(bedP + bed_plane + k);
      nbphi = __ldg(bedP + 2 * bed_plane + k);
    }
    // shift the windows and take row r
    R0 = R1; R1 = R2;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      Sx0[v] = Sx1[v]; Sx1[v] = Sx2[v];
      Wm1[v] = Wm2[v]; Wp1[v] = Wp2[v];
    }
    {
      const T vb = nbv, vh = nhv, vqx = nqxv, vqy = nqyv;
      if (s + 1 < nsteps) {
        if (!CG || (colv && (!EDGE || (r + 1 >= 0 && r + 1 < nx)))) {
          const size_t k = (size_t)(r + 1) * ny + cj;
          nbv = bP[k]; nhv = hP[k]; nqxv = qxP[k]; nqyv = qyP[k];
        } else {
          nbv = T(0); nhv = T(0); nqxv = T(0); nqyv = T(0);
        }
      }
      const T hinv = kp_hinv(vh, p.eps_kp);
      R2.b = vb;
      R2.h = vh;
      R2.hinv = hinv;
      if (RECON == ZB_RECON_ETA) {
        R2.w1 = vb + vh;
        R2.w2 = vqx * hinv;
        R2.w3 = vqy * hinv;
      } else {
        R2.w1 = vh;
        R2.w2 = vqx;
        R2.w3 = vqy;
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        if (v == 0 && BED) continue;   // b's windows feed only its slope
        const T w = R2.w(v);
        const T wl = shu(w), wr = shd(w);
        Wm2[v] = wl;
        Wp2[v] = wr;
        Sx2[v] = (wl + w) + wr;
      }
    }
    if (s < 2) continue;
    // limited slopes of row r-1
    {
      T phi[4], gxa[4], gya[4];
      if constexpr (PAIR) {
        // the x and y components of each variable as the two lanes of
        // paired float32 arithmetic (gradient, limiter increments, bounds)
        const bool clipmin = p.limiter != ZB_LIM_NONE && p.limiter != ZB_LIM_VENKATAKRISHNAN;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          if (v == 0 && BED) {
            gxa[0] = bgx;
            gya[0] = bgy;
            phi[0] = bphi;
            continue;
          }
          const float u = R1.w(v);
          const float tc = (R0.w(v) + R1.w(v)) + R2.w(v);
          const float tl = shu(tc), tr = shd(tc);
          const float2 gv = mul2(sub2(f2(Sx2[v], tr), f2(Sx0[v], tl)), f2(p.inv6dx, p.inv6dy));
          const float wp0 = R2.w(v), wm0 = R0.w(v), w0p = Wp1[v], w0m = Wm1[v];
          const float umax = fmx3(u, wp0, fmx3(wm0, w0p, w0m));
          const float umin = fmn3(u, wp0, fmn3(wm0, w0p, w0m));
          const float2 dd = sub2(f2(umax, umin), f2(u, u));          // (dpos, dneg)
          gxa[v] = gv.x;
          gya[v] = gv.y;
          if (clipmin) {
            const float2 ac = mul2(gv, f2(p.half_dx, p.half_dy));
            phi[v] = phi_clipmin(ac.x, ac.y, dd.x, dd.y);
          } else {
            phi[v] = limiter_phi(p.limiter, gv.x, gv.y, p.half_dx, p.half_dy, dd.x, dd.y,
                                 p.vk_eps2);
          }
        }
      } else {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        if (v == 0 && BED) {   // float64 interior items: the prepared planes
          gxa[0] = bgx;
          gya[0] = bgy;
          phi[0] = bphi;
          continue;
        }
        const T u = R1.w(v);
        const T tc = (R0.w(v) + R1.w(v)) + R2.w(v);
        const T tl = shu(tc), tr = shd(tc);
        const T gx = (Sx2[v] - Sx0[v]) * p.inv6dx;
        const T gy = (tr - tl) * p.inv6dy;
        const T wp0 = R2.w(v), wm0 = R0.w(v), w0p = Wp1[v], w0m = Wm1[v];
        const T umax = fmx3(u, wp0, fmx3(wm0, w0p, w0m));
        const T umin = fmn3(u, wp0, fmn3(wm0, w0p, w0m));
        gxa[v] = gx;
        gya[v] = gy;
        phi[v] = limiter_phi(p.limiter, gx, gy, p.half_dx, p.half_dy, umax - u, umin - u,
                             p.vk_eps2);
      }
      }
      if (CG) {
        // row r-1 = m: boundary cells (stage_tile phase B, non-interior
        // branch) and ghosts (zero slopes); a column-EDGE item's rows are
        // never boundary rows
        const int m = r - 1;
        const bool cellv = colv && (!EDGE || (m >= 0 && m < nx));
        const bool bxl = EDGE && m == 0, bxh = EDGE && m == nx - 1;
        const bool byl = cj == 0, byh = cj == ny - 1;
        const bool bnd = cellv && (bxl || bxh || byl || byh);
        if (!PRE && __any_sync(0xffffffffu, bnd)) {   // PRE: the pre-pass slots
          const int cls = (bxl ? 0 : (bxh ? 2 : 1)) * 3 + (byl ? 0 : (byh ? 2 : 1));
          const T* wx = p.lsq.w[cls][0];
          const T* wy = p.lsq.w[cls][1];
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const T am = shu(R0.w(v)), ap = shd(R0.w(v));
            if (bnd) {
              const T u = R1.w(v);
              T gx = T(0), gy = T(0), umax = u, umin = u;
              T gxv = u, gyv = u;
              if ((bxl || bxh) && p.bc[bxl ? 0 : 1] == ZB_BC_WALL && v == 2) gxv = -u;
              if ((byl || byh) && p.bc[byl ? 2 : 3] == ZB_BC_WALL && v == 3) gyv = -u;
              if ((bxl || bxh) && (byl || byh)) {
                // corner: the class weights (the pseudo-inverse is not diagonal)
                const T nbr[8] = {am, R0.w(v), ap, Wm1[v], Wp1[v], Wm2[v], R2.w(v), Wp2[v]};
                int k = 0;
#pragma unroll
                for (int a = -1; a <= 1; ++a) {
#pragma unroll
                  for (int bb = -1; bb <= 1; ++bb) {
                    if (a == 0 && bb == 0) continue;
                    const bool okn = m + a >= 0 && m + a < nx && cj + bb >= 0 && cj + bb < ny;
                    const T d = okn ? nbr[k] - u : T(0);
                    gx += wx[k] * d;
                    gy += wy[k] * d;
                    ++k;
                  }
                }
                { const T d = gxv - u; gx += wx[8] * d; gy += wy[8] * d; }
                { const T d = gyv - u; gx += wx[9] * d; gy += wy[9] * d; }
              } else if (byl || byh) {
                // side column: the five in-domain neighbours give x the normal
                // matrix diag(4 dx^2, 3 dy^2); y adds its ghost: diag(4 dx^2,
                // 4 dy^2) -- the class weights in closed form
                const T n0 = byl ? ap : am, n1 = byl ? Wp1[v] : Wm1[v];
                const T n2 = byl ? Wp2[v] : Wm2[v];
                gx = ((R2.w(v) + n2) - (R0.w(v) + n0)) * p.inv4dx;
                const T sn = (n0 + n1) + n2;
                gy = (byl ? (sn - gyv) - T(2) * u : (gyv + T(2) * u) - sn) * p.inv4dy;
              } else {
                // side row: the same with the roles of x and y exchanged
                const T n0 = bxl ? Wm2[v] : am, n1 = bxl ? R2.w(v) : R0.w(v);
                const T n2 = bxl ? Wp2[v] : ap;
                gy = ((Wp1[v] + n2) - (Wm1[v] + n0)) * p.inv4dy;
                const T sn = (n0 + n1) + n2;
                gx = (bxl ? (sn - gxv) - T(2) * u : (gxv + T(2) * u) - sn) * p.inv4dx;
              }
              if (!bxh) { umax = fmx(umax, R2.w(v)); umin = fmn(umin, R2.w(v)); }
              if (!bxl) { umax = fmx(umax, R0.w(v)); umin = fmn(umin, R0.w(v)); }
              if (!byh) { umax = fmx(umax, Wp1[v]); umin = fmn(umin, Wp1[v]); }
              if (!byl) { umax = fmx(umax, Wm1[v]); umin = fmn(umin, Wm1[v]); }
              if (bxl || bxh) { const T gg = T(2) * gxv - u; umax = fmx(umax, gg); umin = fmn(umin, gg); }
              if (byl || byh) { const T gg = T(2) * gyv - u; umax = fmx(umax, gg); umin = fmn(umin, gg); }
              gxa[v] = gx;
              gya[v] = gy;
              phi[v] = limiter_phi(p.limiter, gx, gy, p.half_dx, p.half_dy, umax - u, umin - u,
                                   p.vk_eps2);
            }
          }
        }
        if (!cellv) {
#pragma unroll
          for (int v = 0; v < 4; ++v) { phi[v] = T(0); gxa[v] = T(0); gya[v] = T(0); }
        }
      }
      if (RECON == ZB_RECON_ETA) {
        if (p.eps_wet >= T(0) && R1.h < p.eps_wet) {
          phi[0] = phi[1] = phi[2] = phi[3] = T(0);
        }
        phi[0] = zmin(phi[0], phi[1]);
        phi[2] = zmin(phi[2], phi[1]);
        phi[3] = zmin(phi[3], phi[1]);
      }
#pragma unroll
      for (int v = 0; v < 8; ++v) slA[v] = slB[v];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        if constexpr (PAIR) {
          const float2 sv = mul2(f2(phi[v], phi[v]), f2(gxa[v], gya[v]));
          slB[v] = sv.x;
          slB[4 + v] = sv.y;
        } else {
          slB[v] = phi[v] * gxa[v];
          slB[4 + v] = phi[v] * gya[v];
        }
      }
      if constexpr (PRE) {
        // the boundary column's cell of row r - 1 (pre-pass slot r - 1 - (r0 - 1))
        if (cj == 0 || cj == ny - 1) {
          const T* sl = bs + ((cj == 0 ? 0 : PROWS) + (r - r0)) * 12;
#pragma unroll
          for (int v = 0; v < 8; ++v) slB[v] = sl[v];
        }
      }
    }
    if (s < 3) continue;
    // x-face between rows r-2 (A, lower) and r-1 (B, upper)
    T Fh, Fy, fxl_n, fxr_n, Gh, Gx, fyl_t, fyr_own;
    {
      if constexpr (PAIR) {
        const NextRow nv = next_row(R0, slA);
        faces_pair(R0, R1, slA, slB, nv, p, Fh, Fy, fxl_n, fxr_n, Gh, Gx, fyl_t, fyr_own);
        if (s == 3) {          // face r0 - 1/2: only the next row needs it
          fxh_p = Fh; fxt_p = Fy; fxr_p = fxr_n;
          continue;
        }
        if constexpr (PRE) {
          // the y-face on the boundary (the lane below column 0, or column
          // ny - 1) of row r - 2: pre-pass slot r - 2 - (r0 - 1)
          if (cj == -1 || cj == ny - 1) {
            const T* fo = bs + ((cj == -1 ? 0 : PROWS) + (r - 1 - r0)) * 12 + 8;
            Gh = fo[0]; Gx = fo[1]; fyl_t = fo[2]; fyr_own = fo[3];
          }
        } else if (EK >= 2 && (cj == -1 || cj == ny - 1)) {
          // the y-face on the boundary (the lane below column 0, or column
          // ny - 1): the owner's trace against its ghost with normal sign sgy,
          // as the EDGE body evaluates it
          RowW<T> nb;
          nb.b = nv.b; nb.w1 = nv.w1; nb.w2 = nv.w2; nb.w3 = nv.w3; nb.h = nv.h; nb.hinv = T(0);
          const T sln[4] = {nv.s4, nv.s5, nv.s6, nv.s7};
          Side<T> C, D;
          strip_trace<T, RECON>(R0, slA + 4, p.half_dy, C);
          strip_trace<T, RECON>(nb, sln, -p.half_dy, D);
          const bool ylo = cj == -1;
          const Side<T> YL = ylo ? D : C;
          Side<T> YR = YL;
          if (p.bc[ylo ? 2 : 3] == ZB_BC_WALL) {
            YR.qy = -YL.qy;
            YR.uy = -YL.uy;
          }
          const T sgy = ylo ? T(-1) : T(1);
          T Gy, Em, Ep;
          riemann<T, RIEMANN, 1>(YL, YR, sgy, g, Gh, Gx, Gy, Em, Ep);
          const T cesC = half * g * (R0.h + C.h) * (C.b - R0.b);
          const T cesD = -(half * g * (nb.h + D.h) * (D.b - nb.b));
          const T own_n = Gy + Em * sgy + (ylo ? -cesD : cesC) * sgy;
          if (ylo) {
            Gh = -Gh; Gx = -Gx; fyr_own = own_n; fyl_t = T(0);
          } else {
            fyl_t = own_n; fyr_own = T(0);
          }
        }
      } else {
      T Fx, Dm, Dp;
      Side<T> A, B;
      strip_trace<T, RECON>(R0, slA, p.half_dx, A);
      strip_trace<T, RECON>(R1, slB, -p.half_dx, B);
      // EDGE: a face on the x boundary takes the owner's trace (row 0 below
      // the face, row nx-1 above it) against its ghost with normal sign sg
      // (stage_tile's x-face boundary branch)
      const bool xb = EDGE && (r - 1 == 0 || r - 2 == nx - 1);
      const bool xlo = EDGE && r - 1 == 0;
      T sgx = T(1);
      Side<T> L = A, R = B;
      if (xb) {
        L = xlo ? B : A;
        R = L;
        if (p.bc[xlo ? 0 : 1] == ZB_BC_WALL) {
          R.qx = -L.qx;
          R.ux = -L.ux;
        }
        sgx = xlo ? T(-1) : T(1);
      }
      riemann<T, RIEMANN, 0>(L, R, sgx, g, Fh, Fx, Fy, Dm, Dp);
      const T cesA = half * g * (R0.h + A.h) * (A.b - R0.b);
      const T cesB = -(half * g * (R1.h + B.h) * (B.b - R1.b));
      fxl_n = Fx + Dm + cesA;
      fxr_n = -Fx + Dp + cesB;
      if (xb) {
        const T own_n = Fx + Dm * sgx + (xlo ? -cesB : cesA) * sgx;
        if (xlo) {
          Fh = -Fh; Fy = -Fy; fxr_n = own_n; fxl_n = T(0);
        } else {
          fxl_n = own_n; fxr_n = T(0);
        }
      }
      if (s == 3) {            // face r0 - 1/2: only the next row needs it
        fxh_p = Fh; fxt_p = Fy; fxr_p = fxr_n;
        continue;
      }
      // y-faces of row r-2: this lane's top face, the lower lane's one below
      Side<T> C, D;
      T Gy, Em, Ep;
      RowW<T> nb;
      nb.b = shd(R0.b); nb.w1 = shd(R0.w1); nb.w2 = shd(R0.w2); nb.w3 = shd(R0.w3);
      nb.h = shd(R0.h); nb.hinv = shd(R0.hinv);
      T sln[8];
#pragma unroll
      for (int v = 0; v < 4; ++v) sln[4 + v] = shd(slA[4 + v]);
      strip_trace<T, RECON>(R0, slA + 4, p.half_dy, C);
      strip_trace<T, RECON>(nb, sln + 4, -p.half_dy, D);
      // EDGE: a face on the y boundary takes the owner's trace (the next
      // lane's cell 0, or this lane's cell ny-1) against its ghost
      const bool yb = CG && (cj == -1 || cj == ny - 1);
      const bool ylo = CG && cj == -1;
      T sgy = T(1);
      Side<T> YL = C, YR = D;
      if (CG) {
        YL.b = ylo ? D.b : C.b; YL.h = ylo ? D.h : C.h; YL.qx = ylo ? D.qx : C.qx;
        YL.qy = ylo ? D.qy : C.qy; YL.ux = ylo ? D.ux : C.ux; YL.uy = ylo ? D.uy : C.uy;
        const bool wall = yb && p.bc[ylo ? 2 : 3] == ZB_BC_WALL;
        YR.b = yb ? YL.b : D.b; YR.h = yb ? YL.h : D.h; YR.qx = yb ? YL.qx : D.qx;
        YR.ux = yb ? YL.ux : D.ux;
        YR.qy = yb ? (wall ? -YL.qy : YL.qy) : D.qy;
        YR.uy = yb ? (wall ? -YL.uy : YL.uy) : D.uy;
        sgy = ylo ? T(-1) : T(1);
      }
      riemann<T, RIEMANN, 1>(YL, YR, sgy, g, Gh, Gx, Gy, Em, Ep);
      const T cesC = half * g * (R0.h + C.h) * (C.b - R0.b);
      const T cesD = -(half * g * (nb.h + D.h) * (D.b - nb.b));
      fyl_t = Gy + Em + cesC;
      fyr_own = -Gy + Ep + cesD;
      if (yb) {
        const T own_n = Gy + Em * sgy + (ylo ? -cesD : cesC) * sgy;
        if (ylo) {
          Gh = -Gh; Gx = -Gx; fyr_own = own_n; fyl_t = T(0);
        } else {
          fyl_t = own_n; fyr_own = T(0);
        }
      }
      }
      const T fyh_b = shu(Gh), fyt_b = shu(Gx), fyr_b = shu(fyr_own);
      // update of row r-2
      const T kx = p.kx, ky = p.ky;
      const T dh = -(kx * (Fh - fxh_p) + ky * (Gh - fyh_b));
      const T dqx = -(kx * (fxl_n + fxr_p) + ky * (Gx - fyt_b));
      const T dqy = -(kx * (Fy - fxt_p) + ky * (fyl_t + fyr_b));
      fxh_p = Fh; fxt_p = Fy; fxr_p = fxr_n;
      if (!upd) continue;
      const size_t k = (size_t)ro * ny + cj;
      const T hk = R0.h;
      if (RECON != ZB_RECON_ETA) {
        qxk = R0.w2;
        qyk = R0.w3;
      }
      T hn, qxn, qyn;
      if (MODE == MODE_STEP1) {
        hn = hk + dt * dh;
        qxn = qxk + dt * dqx;
        qyn = qyk + dt * dqy;
      } else {
        const T h2 = hk + dt * dh, qx2 = qxk + dt * dqx, qy2 = qyk + dt * dqy;
        hn = half * (h0 + h2);
        qxn = half * (qx0 + qx2);
        qyn = half * (qy0 + qy2);
        if (p.manning_n != T(0)) {
          const T hi0 = kp_hinv(h0, p.eps_kp);
          const T qn = asqrt(qxn * qxn + qyn * qyn);
          const T kf = (-p.g) * (p.manning_n * p.manning_n) * qn * (hi0 * hi0) * cbrt(hi0);
          if (p.implicit_source) {
            const T den = T(1) + dt * (-kf);
            qxn = qxn / den;
            qyn = qyn / den;
          } else {
            qxn = qxn + dt * (qxn * kf);
            qyn = qyn + dt * (qyn * kf);
          }
        }
      }
      hO[k] = hn;
      qxO[k] = qxn;
      qyO[k] = qyn;
      // troubled: h < 0 or a non-finite value (one non-finite term makes
      // the sum's difference with itself NaN; finite states that overflow
      // the sum, |q| ~ 1e38, would flag too)
      const T chk = (hn + qxn) + (qyn + R0.b);
      bad = bad || !(hn >= T(0)) || !(chk - chk == T(0));
      if (MODE == MODE_STEP2) {
        const T hi = kp_hinv(hn, p.eps_kp);
        const T c = asqrt(g * fmx(hn, T(0)));
        const T lx = fabs(qxn * hi) + c, ly = fabs(qyn * hi) + c;
        amax_loc = nmax(amax_loc, nmax(lx, ly));
      }
    }
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(&ctrl->status, (unsigned)ZB_ST_TROUBLED);
  if (MODE == MODE_STEP2) {
    for (int o = 16; o > 0; o >>= 1)
      amax_loc = nmax(amax_loc, __shfl_xor_sync(0xffffffffu, amax_loc, o));
    if (lane == 0) atomic_max_pos_double(&ctrl->amax[(phase + 1) % 3], (double)amax_loc);
  }
}

// Full-coverage item list of a grid with nx, ny >= 4 (strips of SW columns
// from column 0, rows from 0).  Every strip has two EDGE items for the
// boundary rows [0, 2) and [nx - 2, nx).  The rows between go in chunks: SX
// rows for the middle strips (lanes 28 s - 2 .. 28 s + 29 inside the grid,
// the interior body), sxc rows for the strips whose lanes reach outside the
// grid (the first, and the last one or two: the column-EDGE body).  Order:
// the column-EDGE items, the EDGE items (these two kinds form the boundary
// launch), then the interior items.  Item 0 keeps the control block.  Returns
// the item count (item = -1), the count of boundary-launch items (item = -2),
// or with item >= 0 fills its strip, rows and kind (the strip_item EK).
// Column-EDGE chunk heights (B200, 2048^2 and the 512-instance ensemble): a
// single grid's boundary launch shares the SMs with one wave of interior
// items and fills their tail best with short chunks (8 rows: 0.189 ms per
// step; 16: 0.213; 32: 0.261); the ensemble's persistent launches walk their
// longest-first lists one after another and lose less to halo rows with 32
// (2.094 ms per step; 8: 2.21; 16: 2.127; 64: 2.136).
constexpr int SXC_GRID = 8;
constexpr int SXC_ENS = 32;
static_assert(SXC_GRID <= SXC_MAX && SXC_ENS <= SXC_MAX, "column-EDGE pre-pass rows");
__host__ __device__ inline int full_items(int nx, int ny, int item, int* strip, int* r0,
                                          int* r1, int* kind, int sxc, int sx = SX) {
  const int SXC = sxc;
  const int SX = sx;
  const int ns = (ny + SW - 1) / SW;
  // middle strips: 1 <= s <= mh
  int mh = ny >= 30 ? (ny - 30) / SW : 0;
  if (mh > ns - 1) mh = ns - 1;
  const int nmid = mh, nedge = ns - nmid;
  const int nci = nx > 4 ? (nx - 4 + SX - 1) / SX : 0;
  const int ncc = nx > 4 ? (nx - 4 + SXC - 1) / SXC : 0;
  const int nside = nedge * ncc + 2 * ns;
  const int total = nside + nmid * nci;
  if (item == -2) return nside;
  if (item < 0) return total;
  int st, a, b, k;
  if (item < nedge * ncc) {
    const int e = item / ncc;                // edge strips: 0, mh + 1, ..., ns - 1
    st = e == 0 ? 0 : mh + e;
    a = 2 + (item % ncc) * SXC;
    b = a + SXC < nx - 2 ? a + SXC : nx - 2;
    k = 2;
  } else if ((item -= nedge * ncc) < 2 * ns) {
    st = item >> 1;
    a = (item & 1) ? nx - 2 : 0;
    b = a + 2;
    k = 1;
  } else {
    item -= 2 * ns;
    st = 1 + item % nmid;
    a = 2 + (item / nmid) * SX;
    b = a + SX < nx - 2 ? a + SX : nx - 2;
    k = 0;
  }
  *strip = st;
  *r0 = a;
  *r1 = b;
  *kind = k;
  return total;
}

// KIND 0: the interior strips of a grid with a periodic side (the tile kernel
// takes the frame); KIND 1: the boundary items of a full-coverage list
// (column-EDGE and EDGE); KIND 2: its interior items; KIND 3: its interior
// items reading the prepared bed planes (p.bed).  Kinds 1 and 2 are
// separate launches (they run side by side on two streams) so that the
// boundary bodies never raise the interior body's register allocation.
// float32: 4 CTAs of 4 warps per SM (128 registers; the paired-face interior
// body spills at 96).
template <typename T, int RECON, int RIEMANN, int MODE, int KIND>
__global__ void __launch_bounds__(STRIP_NT, sizeof(T) == 4 ? 4 : 2)
swe2d_strip_kernel(const T* __restrict__ bP, const T* __restrict__ hP,
                   const T* __restrict__ qxP, const T* __restrict__ qyP,
                   const T* __restrict__ h0P, const T* __restrict__ qx0P,
                   const T* __restrict__ qy0P, T* __restrict__ hO, T* __restrict__ qxO,
                   T* __restrict__ qyO, zb_ctrl* ctrl, int phase, const SweParams<T> p) {
  int item = blockIdx.x * (STRIP_NT / 32) + (threadIdx.x >> 5);
  int strip, r0, r1, kind = 0;
  if (KIND == 0) {
    const int nstrips = (p.fast_j1 - p.fast_j0) / SW;
    if (item >= nstrips * ((p.fast_i1 - p.fast_i0 + SX - 1) / SX)) return;   // warp-uniform
    strip = item % nstrips;
    r0 = p.fast_i0 + (item / nstrips) * SX;
    r1 = min(r0 + SX, p.fast_i1);
  } else {
    const int ne = full_items(p.nx, p.ny, -2, nullptr, nullptr, nullptr, nullptr, SXC_GRID);
    if (KIND == 1 && item >= ne) return;
    if (KIND >= 2) {
      item += ne;
      const int n = full_items(p.nx, p.ny, -1, nullptr, nullptr, nullptr, nullptr, SXC_GRID);
      if (item >= n) return;
    }
    full_items(p.nx, p.ny, item, &strip, &r0, &r1, &kind, SXC_GRID);
  }
  if (KIND == 1) {
    // warp-uniform: the item's kind
    if (kind == 2)
      strip_item<T, RECON, RIEMANN, MODE, 2>(bP, hP, qxP, qyP, h0P, qx0P, qy0P, hO, qxO, qyO,
                                             ctrl, phase, p, strip, r0, r1, item == 0);
    else
      strip_item<T, RECON, RIEMANN, MODE, 1>(bP, hP, qxP, qyP, h0P, qx0P, qy0P, hO, qxO, qyO,
                                             ctrl, phase, p, strip, r0, r1, item == 0);
  } else {
    strip_item<T, RECON, RIEMANN, MODE, 0, KIND == 3>(bP, hP, qxP, qyP, h0P, qx0P, qy0P, hO,
                                                      qxO, qyO, ctrl, phase, p, strip, r0, r1,
                                                      false);
  }
}

// A second stream per device with a fork and a join event: the EDGE launch of
// a full-coverage stage runs on it beside the interior launch.  Each host
// thread has its own (thread_local), so the fork / join records of calls from
// different threads never interleave and a stream capture on one thread never
// pulls in another thread's launches.  Calls from one thread are ordered by
// the host; on the side stream they run in call order, whatever the caller's
// stream.
struct SideStream {
  cudaStream_t s;
  cudaEvent_t fork, join;
};
static int side_stream(SideStream** out) {
  thread_local SideStream ss[32];
  thread_local unsigned made = 0u;
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 32) return ZB_E_UNSUPPORTED;
  if (!(made & (1u << dev))) {
    ZB_CUDA_TRY(cudaStreamCreateWithFlags(&ss[dev].s, cudaStreamNonBlocking));
    ZB_CUDA_TRY(cudaEventCreateWithFlags(&ss[dev].fork, cudaEventDisableTiming));
    ZB_CUDA_TRY(cudaEventCreateWithFlags(&ss[dev].join, cudaEventDisableTiming));
    made |= 1u << dev;
  }
  *out = &ss[dev];
  return ZB_OK;
}

// ── batched ensemble: one persistent launch per stage over all instances ────
// Each instance is an independent Cartesian grid with its own size, spacing,
// Manning coefficient, dt and control block.  The work list holds one item
// per (instance, tile): {instance, i0, j0, first-tile flag}.  A persistent CTA
// walks items with a grid stride; every item is one stage_tile() call with its
// instance's own dt (read from the instance's control slots), so the whole
// ensemble advances one stage per launch.
template <typename T>
struct EnsDesc {
  SweParams<T> p;
  long long q_off;   // element offset of the instance's (4, C) state
  long long ws_off;  // element offset of its (3, C) stage buffer
};

template <typename T, int TX, int ORDER, int RECON, int RIEMANN, int MODE>
__global__ void __launch_bounds__(NT)
ens_stage_kernel(const EnsDesc<T>* __restrict__ desc, const int4* __restrict__ items,
                 T* Q, T* W, zb_ctrl* ctrls, int phase) {
  using S = Smem<T, TX>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& s = *reinterpret_cast<S*>(smem_raw);
  __shared__ double red[NT / 32];
  const int tid = threadIdx.x;
  // items[0].x = the tile item count; the tile items follow the header
  const int n_items = items[0].x;
  items += 1;
  for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
    const int4 w = items[it];
    const EnsDesc<T>* d = desc + w.x;
    const SweParams<T>& p = d->p;
    zb_ctrl* ctrl = ctrls + w.x;
    const size_t C = (size_t)p.nx * p.ny;
    T* q = Q + d->q_off;
    T* ws = W + d->ws_off;
    const int ph = phase, nph = (ph + 1) % 3, nnph = (ph + 2) % 3;
    const double t = ctrl->t[ph];
    double dtd = dt_from_amax(ctrl->amax[ph], t, p.cfl2r, p.den_fac, p.dt_max, p.t_end);
    const bool ok = isfinite(dtd) && dtd > 0.0;
    const bool lead = w.w != 0 && tid == 0;
    __syncthreads();   // the previous item is done with shared memory
    if (MODE == MODE_STEP1 && lead) {
      if (!ok && t < p.t_end) atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
      ctrl->dt = ok ? dtd : 0.0;
      ctrl->t[nph] = ok ? t + dtd : t;
      ctrl->amax[nnph] = 0.0;
    }
    if (!ok) {
      if (MODE == MODE_STEP2 && lead) ctrl->amax[nph] = ctrl->amax[ph];
      continue;   // block-uniform: every thread of the CTA skips this item
    }
    if (MODE == MODE_STEP1) {
      stage_tile<T, TX, ORDER, RECON, RIEMANN, MODE_STEP1>(
          s, red, w.y, w.z, q, q + C, q + 2 * C, q + 3 * C, nullptr, nullptr, nullptr, ws,
          ws + C, ws + 2 * C, ctrl, ph, nullptr, nullptr, nullptr, p, dtd, w.w != 0);
    } else {
      stage_tile<T, TX, ORDER, RECON, RIEMANN, MODE_STEP2>(
          s, red, w.y, w.z, q, ws, ws + C, ws + 2 * C, q + C, q + 2 * C, q + 3 * C, q + C,
          q + 2 * C, q + 3 * C, ctrl, ph, nullptr, nullptr, nullptr, p, dtd, w.w != 0);
    }
  }
}

// One strip item of an instance: stage 1 reads Q and writes the stage buffer,
// stage 2 reads the stage buffer and Q0 = Q and writes Q.
template <typename T, int MODE, int EK>
__device__ __forceinline__ void ens_item(const EnsDesc<T>* d, T* Q, T* W, zb_ctrl* ctrl,
                                         int phase, int strip, int r0, int r1, bool lead) {
  const SweParams<T>& p = d->p;
  const size_t C = (size_t)p.nx * p.ny;
  T* q = Q + d->q_off;
  T* ws = W + d->ws_off;
  if (MODE == MODE_STEP1)
    strip_item<T, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR, MODE_STEP1, EK>(
        q, q + C, q + 2 * C, q + 3 * C, nullptr, nullptr, nullptr, ws, ws + C, ws + 2 * C,
        ctrl, phase, p, strip, r0, r1, lead);
  else
    strip_item<T, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR, MODE_STEP2, EK>(
        q, ws, ws + C, ws + 2 * C, q + C, q + 2 * C, q + 3 * C, q + C, q + 2 * C, q + 3 * C,
        ctrl, phase, p, strip, r0, r1, lead);
}

// All instances' strip items of one body (EK, as strip_item: 0 interior, 1
// EDGE, 3 column EDGE with its pre-pass): persistent warps walk them.  The
// work list's header items[0] = {tile items, interior strip items, EDGE strip
// items, column-EDGE strip items}; the lists follow it in that order.  Each
// body is a launch of its own, so that the boundary bodies' extra live values
// never raise another body's register allocation.
template <typename T, int MODE, int EK>
__global__ void __launch_bounds__(STRIP_NT, sizeof(T) == 4 ? 4 : 2)
ens_strip_kernel(const EnsDesc<T>* __restrict__ desc, const int4* __restrict__ items, T* Q,
                 T* W, zb_ctrl* ctrls, int phase) {
  static_assert(EK == 0 || EK == 1 || EK == 3, "ensemble bodies");
  const int4 hd = items[0];
  const int4* list = items + 1 + hd.x + (EK >= 1 ? hd.y : 0) + (EK == 3 ? hd.z : 0);
  const int n = EK == 0 ? hd.y : (EK == 1 ? hd.z : hd.w);
  const int nw = gridDim.x * (STRIP_NT / 32);
  for (int it = blockIdx.x * (STRIP_NT / 32) + (threadIdx.x >> 5); it < n; it += nw) {
    // w = {instance, strip, r0, flags | r1 << 3}; flags bit 1 = the item keeps
    // the instance's control block
    const int4 w = list[it];
    ens_item<T, MODE, EK>(desc + w.x, Q, W, ctrls + w.x, phase, w.y, w.z, w.w >> 3,
                          (w.w & 2) != 0);
  }
}

template <typename T>
__global__ void __launch_bounds__(NT)
ens_amax_kernel(const EnsDesc<T>* __restrict__ desc, const T* __restrict__ Q, zb_ctrl* ctrls,
                int n_inst, int phase, double t0, T g, T eps) {
  __shared__ double red[NT / 32];
  for (int i = blockIdx.x; i < n_inst; i += gridDim.x) {
    const EnsDesc<T>* d = desc + i;
    const size_t C = (size_t)d->p.nx * d->p.ny;
    const T* q = Q + d->q_off;
    double m = 0.0;
    for (size_t k = threadIdx.x; k < C; k += NT) {
      const T h = q[C + k];
      const T hi = kp_hinv(h, eps);
      const T c = asqrt(g * nmax(h, T(0)));
      m = nmax(m, (double)nmax(fabs(q[2 * C + k] * hi) + c, fabs(q[3 * C + k] * hi) + c));
    }
    __syncthreads();
    m = block_max_double(m, red);
    if (threadIdx.x == 0) {
      zb_ctrl* ctrl = ctrls + i;
      for (int j = 0; j < 3; ++j) { ctrl->amax[j] = 0.0; ctrl->t[j] = 0.0; }
      ctrl->amax[phase] = m;
      ctrl->t[phase] = t0;
      ctrl->dt = 0.0;
      ctrl->status = 0u;
      ctrl->steps = 0u;
      ctrl->troubled = 0u;
    }
  }
}

// ── wave-speed max / aux / mass kernels ─────────────────────────────────────
template <typename T>
__global__ void __launch_bounds__(NT)
swe2d_amax_kernel(const T* __restrict__ hP, const T* __restrict__ qxP,
                  const T* __restrict__ qyP, size_t C, T g, T eps_kp,
                  double* out) {
  __shared__ double red[NT / 32];
  double m = 0.0;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C;
       k += (size_t)gridDim.x * NT) {
    const T h = hP[k];
    const T hi = kp_hinv(h, eps_kp);
    const T c = asqrt(g * nmax(h, T(0)));
    const T lx = fabs(qxP[k] * hi) + c, ly = fabs(qyP[k] * hi) + c;
    m = nmax(m, (double)nmax(lx, ly));
  }
  m = block_max_double(m, red);
  if (threadIdx.x == 0) atomic_max_pos_double(out, m);
}

// The bed's interior least-squares gradient and limiter value, one thread per
// cell: the slope block of strip_item for variable 0 (b) -- the float32
// paired block, the float64 scalar one -- in the same operations and order
// ((left + centre) + right sums, difference and scaling, three-input bounds,
// the limiter), so the strip body that reads these planes produces the same
// bits as the one that evaluates them.  Cells on the domain boundary get zeros
// (the interior body never reads them; boundary cells take the boundary
// classes).
template <typename T>
__global__ void __launch_bounds__(NT)
swe2d_bed_kernel(const T* __restrict__ b, T* __restrict__ bed, const SweParams<T> p) {
  const int nx = p.nx, ny = p.ny;
  const size_t n = (size_t)nx * ny;
  const bool clipmin = p.limiter != ZB_LIM_NONE && p.limiter != ZB_LIM_VENKATAKRISHNAN;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(k / (size_t)ny), j = (int)(k % (size_t)ny);
    T gx = T(0), gy = T(0), phi = T(0);
    if (i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1) {
      const T* rm = b + (k - ny);   // row i - 1
      const T* rc = b + k;          // row i
      const T* rp = b + (k + ny);   // row i + 1
      const T u = rc[0];
      const T sx0 = (rm[-1] + rm[0]) + rm[1];   // row sums of rows i -/+ 1
      const T sx2 = (rp[-1] + rp[0]) + rp[1];
      const T tl = (rm[-1] + rc[-1]) + rp[-1];  // column sums of columns j -/+ 1
      const T tr = (rm[1] + rc[1]) + rp[1];
      const T umax = fmx3(u, rp[0], fmx3(rm[0], rc[1], rc[-1]));
      const T umin = fmn3(u, rp[0], fmn3(rm[0], rc[1], rc[-1]));
      if constexpr (std::is_same<T, float>::value) {
        const float2 gv = mul2(sub2(f2(sx2, tr), f2(sx0, tl)), f2(p.inv6dx, p.inv6dy));
        const float2 dd = sub2(f2(umax, umin), f2(u, u));
        gx = gv.x;
        gy = gv.y;
        if (clipmin) {
          const float2 ac = mul2(gv, f2(p.half_dx, p.half_dy));
          phi = phi_clipmin(ac.x, ac.y, dd.x, dd.y);
        } else {
          phi = limiter_phi(p.limiter, gv.x, gv.y, p.half_dx, p.half_dy, dd.x, dd.y, p.vk_eps2);
        }
      } else {
        gx = (sx2 - sx0) * p.inv6dx;
        gy = (tr - tl) * p.inv6dy;
        phi = limiter_phi(p.limiter, gx, gy, p.half_dx, p.half_dy, umax - u, umin - u, p.vk_eps2);
      }
    }
    bed[k] = gx;
    bed[n + k] = gy;
    bed[2 * n + k] = phi;
  }
}

__global__ void swe2d_ctrl_init_kernel(zb_ctrl* ctrl, int phase, double t0) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) { ctrl->amax[i] = 0.0; ctrl->t[i] = 0.0; }
    ctrl->t[phase] = t0;
    ctrl->dt = 0.0;
    ctrl->status = 0u;
    ctrl->steps = 0u;
    ctrl->troubled = 0u;
  }
}

__global__ void swe2d_dt_finalize_kernel(zb_ctrl* ctrl, double t, double cfl2r,
                                         double den_fac, double dt_max,
                                         double t_end) {
  if (threadIdx.x == 0) {
    const double dt = dt_from_amax(ctrl->reserved[0], t, cfl2r, den_fac, dt_max, t_end);
    ctrl->dt = dt;
    if (!(isfinite(dt) && dt > 0.0) && t < t_end)
      atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
  }
}

__global__ void zero_double_kernel(double* p) { *p = 0.0; }

// LSQ derivative aux rows with extrapolation ghosts (delta 0)
template <typename T>
__global__ void __launch_bounds__(NT)
swe2d_aux_kernel(const T* __restrict__ Q, T* __restrict__ A, int nx, int ny,
                 T eps_kp, const LsqTable<T> lsq) {
  const size_t C = (size_t)nx * ny;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C;
       k += (size_t)gridDim.x * NT) {
    const int gi = (int)(k / ny), gj = (int)(k - (size_t)gi * ny);
    const bool bxl = gi == 0, bxh = gi == nx - 1, byl = gj == 0, byh = gj == ny - 1;
    const int cls = (bxl ? 0 : (bxh ? 2 : 1)) * 3 + (byl ? 0 : (byh ? 2 : 1));
    const T* wx = lsq.w[cls][0];
    const T* wy = lsq.w[cls][1];
    T g[4][2];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const T* U = Q + (size_t)v * C;
      const T u = U[k];
      T gx = T(0), gy = T(0);
      int s = 0;
      for (int a = -1; a <= 1; ++a)
        for (int bb = -1; bb <= 1; ++bb) {
          if (a == 0 && bb == 0) continue;
          const bool ok = gi + a >= 0 && gi + a < nx && gj + bb >= 0 && gj + bb < ny;
          const T d = ok ? U[k + (long long)a * ny + bb] - u : T(0);
          gx += wx[s] * d;
          gy += wy[s] * d;
          ++s;
        }
      g[v][0] = gx;
      g[v][1] = gy;
    }
    A[0 * C + k] = g[2][0];
    A[1 * C + k] = g[1][0];
    A[2 * C + k] = g[3][1];
    A[3 * C + k] = g[1][1];
    A[4 * C + k] = g[0][0];
    A[5 * C + k] = g[0][1];
    A[6 * C + k] = kp_hinv(Q[C + k], eps_kp);
  }
}

template <typename T>
__global__ void __launch_bounds__(NT)
mass_partial_kernel(const T* __restrict__ h, size_t C, double vol, double* partial) {
  __shared__ double red[NT];
  double acc = 0.0;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C;
       k += (size_t)gridDim.x * NT)
    acc += (double)h[k] * vol;
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void mass_final_kernel(const double* partial, int n, zb_ctrl* ctrl) {
  __shared__ double red[NT];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += NT) acc += partial[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) ctrl->mass = red[0];
}

// Manning friction as RK1 with a given aux hinv0 (ode.py:14-18,
// solver_jax.py:373-397, 1129); implicit = point-implicit closed form
template <typename T>
__global__ void __launch_bounds__(NT)
swe2d_source_kernel(T* __restrict__ qx, T* __restrict__ qy, const T* __restrict__ hinv0,
                    size_t C, T g, T n, T dt, int implicit) {
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C;
       k += (size_t)gridDim.x * NT) {
    const T hi0 = hinv0[k];
    T a = qx[k], b = qy[k];
    const T qn = asqrt(a * a + b * b);
    const T kf = (-g) * (n * n) * qn * (hi0 * hi0) * cbrt(hi0);
    if (implicit) {
      const T den = T(1) + dt * (-kf);
      a = a / den;
      b = b / den;
    } else {
      a = a + dt * (a * kf);
      b = b + dt * (b * kf);
    }
    qx[k] = a;
    qy[k] = b;
  }
}

// the float64 quotient, square root and reciprocal square root of the
// kernels above, for their accuracy test (zb_newton_check_f64)
__global__ void __launch_bounds__(NT)
newton_check_kernel(const double* __restrict__ a, const double* __restrict__ b,
                    double* __restrict__ out, long long n) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n;
       k += (long long)gridDim.x * NT) {
    out[k] = ndiv(a[k], b[k]);
    out[n + k] = nsqrt(b[k]);
    out[2 * n + k] = nrsqrt(b[k]);
  }
}

// ── host side ───────────────────────────────────────────────────────────────
constexpr int MASS_BLOCKS = 1184;   // 148 SMs x 8

static bool valid_cfg(const zb_swe2d_cfg* c) {
  if (!c) return false;
  if (c->nx < 3 || c->ny < 3) return false;
  if ((long long)c->nx * c->ny > (1LL << 31)) return false;
  if (!(c->dx > 0 && c->dy > 0)) return false;
  if (c->order != 1 && c->order != 2) return false;
  if (c->recon < 0 || c->recon > 2 || c->riemann < 0 || c->riemann > 2) return false;
  if (c->limiter < 0 || c->limiter > 3) return false;
  for (int i = 0; i < 4; ++i)
    if (c->bc[i] < 0 || c->bc[i] > 2) return false;
  if ((c->bc[0] == ZB_BC_PERIODIC) != (c->bc[1] == ZB_BC_PERIODIC)) return false;
  if ((c->bc[2] == ZB_BC_PERIODIC) != (c->bc[3] == ZB_BC_PERIODIC)) return false;
  if (c->dtype != ZB_F32 && c->dtype != ZB_F64) return false;
  if (c->order == 1 && c->recon != ZB_RECON_CONSTANT) return false;
  if (c->order == 2 && c->recon == ZB_RECON_CONSTANT) return false;
  if (c->dim_factor < 1 || c->degree < 0) return false;
  return true;
}

// Least-squares weights of the 9 Cartesian cell classes: pseudo-inverse of the
// offsets of the in-domain 3x3 neighbours plus, per derivative direction, the
// ghost of the boundary face normal to that direction (oracle/mesh.py,
// _lsq_weights; pinned against the reference's derivative aux rows).
template <typename T>
static LsqTable<T> make_lsq(double dx, double dy) {
  LsqTable<T> tab;
  std::memset(&tab, 0, sizeof(tab));
  for (int ci = 0; ci < 3; ++ci)
    for (int cj = 0; cj < 3; ++cj) {
      const int cls = ci * 3 + cj;
      for (int d = 0; d < 2; ++d) {
        double px[10], py[10];
        int slot[10], n = 0, k = 0;
        for (int a = -1; a <= 1; ++a)
          for (int b = -1; b <= 1; ++b) {
            if (a == 0 && b == 0) continue;
            const bool okx = !(ci == 0 && a < 0) && !(ci == 2 && a > 0);
            const bool oky = !(cj == 0 && b < 0) && !(cj == 2 && b > 0);
            if (okx && oky) { px[n] = a * dx; py[n] = b * dy; slot[n] = k; ++n; }
            ++k;
          }
        if (d == 0 && ci != 1) { px[n] = (ci == 0 ? -1.0 : 1.0) * dx; py[n] = 0.0; slot[n] = 8; ++n; }
        if (d == 1 && cj != 1) { px[n] = 0.0; py[n] = (cj == 0 ? -1.0 : 1.0) * dy; slot[n] = 9; ++n; }
        double sxx = 0, sxy = 0, syy = 0;
        for (int m = 0; m < n; ++m) { sxx += px[m] * px[m]; sxy += px[m] * py[m]; syy += py[m] * py[m]; }
        const double det = sxx * syy - sxy * sxy;
        const double i00 = syy / det, i01 = -sxy / det, i11 = sxx / det;
        for (int m = 0; m < n; ++m) {
          const double wxm = i00 * px[m] + i01 * py[m];
          const double wym = i01 * px[m] + i11 * py[m];
          tab.w[cls][d][slot[m]] = (T)(d == 0 ? wxm : wym);
        }
      }
    }
  return tab;
}

// the scheme whose interior body reads prepared bed slopes: order 2, eta
// reconstruction, HLL with hydrostatic reconstruction (float32 or float64)
static bool bed_scheme(const zb_swe2d_cfg* c) {
  return c->order == 2 && c->recon == ZB_RECON_ETA && c->riemann == ZB_RIEMANN_HLL_HR;
}

template <typename T>
static SweParams<T> make_params(const zb_swe2d_cfg* c, double alpha, double beta,
                                double dt_stage = -1.0) {
  SweParams<T> p;
  std::memset(&p, 0, sizeof(p));
  p.nx = c->nx;
  p.ny = c->ny;
  p.half_dx = (T)(0.5 * c->dx);
  p.half_dy = (T)(0.5 * c->dy);
  const double vol = c->dx * c->dy;
  p.kx = (T)(c->dy / vol);
  p.ky = (T)(c->dx / vol);
  p.g = (T)c->g;
  p.eps_kp = (T)c->wet_dry_eps;
  p.eps_wet = (T)(c->eps_wet < 0 ? -1.0 : c->eps_wet);
  p.manning_n = (T)c->manning_n;
  const double hv = std::pow(vol, 0.5);
  p.vk_eps2 = (T)(hv * hv);
  for (int i = 0; i < 4; ++i) p.bc[i] = c->bc[i];
  p.limiter = c->limiter;
  p.implicit_source = c->implicit_source;
  const double r_in = c->dx * c->dy / (c->dx + c->dy);
  p.cfl2r = c->cfl * 2.0 * r_in;
  p.den_fac = (double)c->dim_factor * (double)(2 * c->degree + 1);
  p.dt_max = c->dt_max;
  p.t_end = c->t_end;
  p.alpha = alpha;
  p.beta = beta;
  p.dt_stage = dt_stage;
  p.lsq = make_lsq<T>(c->dx, c->dy);
  p.inv6dx = (T)(1.0 / (6.0 * c->dx));
  p.inv6dy = (T)(1.0 / (6.0 * c->dy));
  p.inv4dx = (T)(1.0 / (4.0 * c->dx));
  p.inv4dy = (T)(1.0 / (4.0 * c->dy));
  p.fast_i0 = p.fast_i1 = p.fast_j0 = p.fast_j1 = 0;
  p.strip_full = 0;
  p.bed = (bed_scheme(c) && (c->dtype == ZB_F64) == std::is_same<T, double>::value)
              ? (const T*)c->bed : nullptr;
  return p;
}

template <typename T>
constexpr int tile_x() { return sizeof(T) == 4 ? 16 : 8; }

// number of frame tiles the tile kernel enumerates when the strip kernel
// owns the interior (see swe2d_stage_kernel)
template <int TX>
static int frame_tiles(int nx, int ny, int fi0, int fi1, int fj0, int fj1) {
  const int ntc = (ny + TY - 1) / TY, ntr = (nx + TX - 1) / TX;
  const int tra = (fi0 + TX - 1) / TX, trb = std::max(tra, fi1 / TX);
  const int tca = (fj0 + TY - 1) / TY, tcb = std::max(tca, fj1 / TY);
  return tra * ntc + (ntr - trb) * ntc + (trb - tra) * (tca + ntc - tcb);
}

template <typename T, int ORDER, int RECON, int RIEMANN, int MODE, int TX = tile_x<T>()>
static int launch_stage(const zb_swe2d_cfg* c, const T* b, const T* h, const T* qx,
                        const T* qy, const T* h0, const T* qx0, const T* qy0,
                        T* ho, T* qxo, T* qyo, zb_ctrl* ctrl, int phase,
                        const SweParams<T>& p, cudaStream_t st,
                        const T* hinv_src = nullptr,
                        const unsigned char* force_o1 = nullptr,
                        unsigned char* trouble_out = nullptr) {
  auto kern = swe2d_stage_kernel<T, TX, ORDER, RECON, RIEMANN, MODE>;
  const size_t sm = sizeof(Smem<T, TX>);
  static std::atomic<unsigned> attr_mask{0u};   // per instantiation, one bit per device
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 32) return ZB_E_UNSUPPORTED;
  if (!(attr_mask.load() & (1u << dev))) {
    ZB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    attr_mask.fetch_or(1u << dev);
  }
  dim3 grid((c->ny + TY - 1) / TY, (c->nx + TX - 1) / TX);
  if (p.fast_i1 > p.fast_i0)
    grid = dim3(frame_tiles<TX>(c->nx, c->ny, p.fast_i0, p.fast_i1, p.fast_j0, p.fast_j1), 1);
  kern<<<grid, NT, sm, st>>>(b, h, qx, qy, h0, qx0, qy0, ho, qxo, qyo, ctrl, phase,
                             hinv_src, force_o1, trouble_out, p);
  return zb_launch_check();
}

// part: -1 = the whole step, 0 = first launch only, 1 = second launch only
template <typename T, int ORDER, int RECON, int RIEMANN>
static int run_step(const zb_swe2d_cfg* c, T* Q, T* ws, zb_ctrl* ctrl, int phase,
                    int part, cudaStream_t st) {
  const size_t C = (size_t)c->nx * c->ny;
  T *b = Q, *h = Q + C, *qx = Q + 2 * C, *qy = Q + 3 * C;
  const SweParams<T> p = make_params<T>(c, 0.0, 1.0);
  T *h1 = ws, *qx1 = ws + C, *qy1 = ws + 2 * C;
  if (ORDER == 1) {
    // Euler reads the stencil of Q and cannot write Q in place: write the
    // workspace (launch 0), then copy the three evolving planes back (part 1)
    if (part != 1) {
      int rc = launch_stage<T, ORDER, RECON, RIEMANN, MODE_EULER>(
          c, b, h, qx, qy, nullptr, nullptr, nullptr, h1, qx1, qy1, ctrl, phase, p, st);
      if (rc) return rc;
    }
    if (part != 0)
      ZB_CUDA_TRY(cudaMemcpyAsync(h, h1, 3 * C * sizeof(T), cudaMemcpyDeviceToDevice, st));
    return ZB_OK;
  }
  // Without a periodic side the strip kernel covers the whole grid (strips
  // and row chunks that reach the boundary take its EDGE body) and keeps the
  // control block.  With one, the interior (two cells in from every side)
  // goes to the strip kernel and the boundary frame to the tile kernel.
  SweParams<T> pf = p;
  int nstrips = 0;
  if (ORDER == 2) {
    bool periodic = false;
    for (int sd = 0; sd < 4; ++sd) periodic = periodic || c->bc[sd] == ZB_BC_PERIODIC;
    if (!periodic && c->nx >= 4 && c->ny >= 4) {
      nstrips = (c->ny + SW - 1) / SW;
      pf.fast_i0 = 0;
      pf.fast_i1 = c->nx;
      pf.fast_j0 = 0;
      pf.fast_j1 = SW * nstrips;
      pf.strip_full = 1;
    } else if (c->ny >= 32 && c->nx >= 8) {
      nstrips = (c->ny - 32) / SW + 1;
      pf.fast_i0 = 2;
      pf.fast_i1 = c->nx - 2;
      pf.fast_j0 = 2;
      pf.fast_j1 = 2 + SW * nstrips;
    }
  }
  const bool strips = pf.fast_i1 > pf.fast_i0;
  const bool tiles = !pf.strip_full;
  const int nitems = !strips ? 0
                     : pf.strip_full ? full_items(c->nx, c->ny, -1, nullptr, nullptr, nullptr,
                                                       nullptr, SXC_GRID)
                                     : nstrips * ((pf.fast_i1 - pf.fast_i0 + SX - 1) / SX);
  const int sgrid = (nitems + STRIP_NT / 32 - 1) / (STRIP_NT / 32);
  // full coverage: the boundary items on the side stream, the interior items here
  SideStream* side = nullptr;
  int ne = 0, ni = 0;
  if (pf.strip_full) {
    int rc = side_stream(&side);
    if (rc) return rc;
    ne = full_items(c->nx, c->ny, -2, nullptr, nullptr, nullptr, nullptr, SXC_GRID);
    ni = nitems - ne;
  }
  const int wpb = STRIP_NT / 32;
  auto launch_strips = [&](auto mode, const T* h_, const T* qx_, const T* qy_, const T* h0_,
                           const T* qx0_, const T* qy0_, T* ho_, T* qxo_, T* qyo_) -> int {
    constexpr int M = decltype(mode)::value;
    if (!pf.strip_full) {
      swe2d_strip_kernel<T, RECON, RIEMANN, M, 0><<<sgrid, STRIP_NT, 0, st>>>(
          b, h_, qx_, qy_, h0_, qx0_, qy0_, ho_, qxo_, qyo_, ctrl, phase, pf);
      return zb_launch_check();
    }
    ZB_CUDA_TRY(cudaEventRecord(side->fork, st));
    ZB_CUDA_TRY(cudaStreamWaitEvent(side->s, side->fork, 0));
    swe2d_strip_kernel<T, RECON, RIEMANN, M, 1><<<(ne + wpb - 1) / wpb, STRIP_NT, 0, side->s>>>(
        b, h_, qx_, qy_, h0_, qx0_, qy0_, ho_, qxo_, qyo_, ctrl, phase, pf);
    ZB_CUDA_TRY(cudaGetLastError());
    if (ni > 0) {
      // the interior items read the prepared bed planes when there are some
      constexpr bool BEDK = RECON == ZB_RECON_ETA &&
                            RIEMANN == ZB_RIEMANN_HLL_HR;
      bool done = false;
      if constexpr (BEDK) {
        if (pf.bed) {
          swe2d_strip_kernel<T, RECON, RIEMANN, M, 3><<<(ni + wpb - 1) / wpb, STRIP_NT, 0, st>>>(
              b, h_, qx_, qy_, h0_, qx0_, qy0_, ho_, qxo_, qyo_, ctrl, phase, pf);
          ZB_CUDA_TRY(cudaGetLastError());
          done = true;
        }
      }
      if (!done) {
        swe2d_strip_kernel<T, RECON, RIEMANN, M, 2><<<(ni + wpb - 1) / wpb, STRIP_NT, 0, st>>>(
            b, h_, qx_, qy_, h0_, qx0_, qy0_, ho_, qxo_, qyo_, ctrl, phase, pf);
        ZB_CUDA_TRY(cudaGetLastError());
      }
    }
    ZB_CUDA_TRY(cudaEventRecord(side->join, side->s));
    ZB_CUDA_TRY(cudaStreamWaitEvent(st, side->join, 0));
    return ZB_OK;
  };
  using M1 = std::integral_constant<int, MODE_STEP1>;
  using M2 = std::integral_constant<int, MODE_STEP2>;
  if (part != 1) {
    if (strips) {
      int rc = launch_strips(M1(), h, qx, qy, nullptr, nullptr, nullptr, h1, qx1, qy1);
      if (rc) return rc;
    }
    if (tiles) {
      // the frame is thin: 8-row tiles waste less of their work on it
      int rc = launch_stage<T, ORDER, RECON, RIEMANN, MODE_STEP1, 8>(
          c, b, h, qx, qy, nullptr, nullptr, nullptr, h1, qx1, qy1, ctrl, phase, pf, st);
      if (rc) return rc;
    }
  }
  if (part == 0) return ZB_OK;
  if (strips) {
    int rc = launch_strips(M2(), h1, qx1, qy1, h, qx, qy, h, qx, qy);
    if (rc) return rc;
  }
  if (!tiles) return ZB_OK;
  return launch_stage<T, ORDER, RECON, RIEMANN, MODE_STEP2, 8>(
      c, b, h1, qx1, qy1, h, qx, qy, h, qx, qy, ctrl, phase, pf, st);
}

template <typename T, int ORDER, int RECON, int RIEMANN>
static int run_generic_stage(const zb_swe2d_cfg* c, const T* Qk, const T* Q0, T* Qo,
                             double alpha, double beta, double dt, zb_ctrl* ctrl,
                             const T* hinv_src, const unsigned char* force_o1,
                             unsigned char* trouble_out, cudaStream_t st) {
  const size_t C = (size_t)c->nx * c->ny;
  const SweParams<T> p = make_params<T>(c, alpha, beta, dt);
  const T* b0 = Q0 ? Q0 : Qk;
  return launch_stage<T, ORDER, RECON, RIEMANN, MODE_STAGE>(
      c, b0, Qk + C, Qk + 2 * C, Qk + 3 * C, Q0 ? Q0 + C : nullptr,
      Q0 ? Q0 + 2 * C : nullptr, Q0 ? Q0 + 3 * C : nullptr, Qo + C, Qo + 2 * C,
      Qo + 3 * C, ctrl, 0, p, st, hinv_src, force_o1, trouble_out);
}

// dispatch over (order, recon, riemann)
template <typename T, typename F>
static int dispatch(const zb_swe2d_cfg* c, F&& f) {
#define ZB_CASE(O, R, M)                                                       \
  if (c->order == O && c->recon == R && c->riemann == M)                       \
    return f(std::integral_constant<int, O>(), std::integral_constant<int, R>(), \
             std::integral_constant<int, M>());
  ZB_CASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_RUSANOV)
  ZB_CASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_RUSANOV_HR)
  ZB_CASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_HLL_HR)
  ZB_CASE(2, ZB_RECON_CONSERVATIVE, ZB_RIEMANN_RUSANOV)
  ZB_CASE(2, ZB_RECON_CONSERVATIVE, ZB_RIEMANN_RUSANOV_HR)
  ZB_CASE(2, ZB_RECON_CONSERVATIVE, ZB_RIEMANN_HLL_HR)
  ZB_CASE(2, ZB_RECON_ETA, ZB_RIEMANN_RUSANOV_HR)
  ZB_CASE(2, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR)
#undef ZB_CASE
  return ZB_E_UNSUPPORTED;
}

template <typename T>
static int amax_into(const zb_swe2d_cfg* c, const T* Q, double* dst, cudaStream_t st) {
  const size_t C = (size_t)c->nx * c->ny;
  zero_double_kernel<<<1, 1, 0, st>>>(dst);
  const int blocks = (int)std::min<size_t>((C + NT - 1) / NT, 148 * 16);
  swe2d_amax_kernel<T><<<blocks, NT, 0, st>>>(Q + C, Q + 2 * C, Q + 3 * C, C, (T)c->g,
                                              (T)c->wet_dry_eps, dst);
  return zb_launch_check();
}


// ── ensemble host side ──────────────────────────────────────────────────────
template <typename T>
static size_t ens_desc_bytes(int n_inst) {
  return ((size_t)n_inst * sizeof(EnsDesc<T>) + 255) / 256 * 256;
}

// strip region of an instance: the whole grid (every instance has wall or
// extrapolation sides), or empty for a grid too small for strips (all tiles)
struct Fast { int i0, i1, j0, j1, nstrips, nchunks; };
static Fast fast_region(int nx, int ny) {
  Fast f{0, 0, 0, 0, 0, 0};
  if (nx >= 4 && ny >= 4) {
    f.nstrips = (ny + SW - 1) / SW;
    f.nchunks = (nx + SX - 1) / SX;
    f.i1 = nx; f.j1 = SW * f.nstrips;
  }
  return f;
}

// strip items of an instance (the single grid's full-coverage list):
// {strip, r0, r1, flags}; flags bit 0 = a boundary-launch item, bit 1 = it
// keeps the control block, bit 2 = a column-EDGE item (else EDGE, when bit 0)
// the chunk heights of an instance's size class (zb_ens_tuning)
static void ens_class_rows(const zb_ens_tuning& t, const zb_ens_instance& in, int* sxc,
                           int* sx) {
  const int side = std::max(in.nx, in.ny);
  int c = 0;
  while (c < t.n_classes - 1 && side > t.class_max_side[c]) ++c;
  *sxc = t.edge_rows[c];
  *sx = t.interior_rows[c];
}

template <typename F>
static void ens_strip_items(const zb_ens_instance& in, const zb_ens_tuning& t, F&& visit) {
  if (fast_region(in.nx, in.ny).nstrips == 0) return;
  int sxc, sx;
  ens_class_rows(t, in, &sxc, &sx);
  const int n = full_items(in.nx, in.ny, -1, nullptr, nullptr, nullptr, nullptr, sxc, sx);
  for (int it = 0; it < n; ++it) {
    int st, r0, r1, kind;
    full_items(in.nx, in.ny, it, &st, &r0, &r1, &kind, sxc, sx);
    visit(st, r0, r1, (kind != 0 ? 1 : 0) | (it == 0 ? 2 : 0) | (kind == 2 ? 4 : 0));
  }
}

// tiles of an instance that the strips do not cover (all of a small grid's)
template <typename F>
static void ens_frame_tiles(const zb_ens_instance& in, int tile_x, F&& visit) {
  if (fast_region(in.nx, in.ny).nstrips > 0) return;
  for (int i0 = 0; i0 < in.nx; i0 += tile_x)
    for (int j0 = 0; j0 < in.ny; j0 += TY) visit(i0, j0);
}

static void ens_counts(const zb_ens_instance* inst, int n, const zb_ens_tuning& t,
                       size_t* tiles, size_t* strips) {
  *tiles = 0;
  *strips = 0;
  for (int i = 0; i < n; ++i) {
    ens_frame_tiles(inst[i], t.tile_x, [&](int, int) { ++*tiles; });
    if (fast_region(inst[i].nx, inst[i].ny).nstrips > 0) {
      int sxc, sx;
      ens_class_rows(t, inst[i], &sxc, &sx);
      *strips += (size_t)full_items(inst[i].nx, inst[i].ny, -1, nullptr, nullptr, nullptr,
                                    nullptr, sxc, sx);
    }
  }
}

// the launch shape of the untuned entry points: one size class, 32-row
// column-EDGE chunks, 64-row interior chunks, 4 (float) or 2 (double) strip
// CTAs per SM
static zb_ens_tuning ens_default_tuning(const zb_swe2d_cfg* c, int tile_x) {
  zb_ens_tuning t;
  std::memset(&t, 0, sizeof(t));
  t.tile_x = tile_x;
  t.ctas_per_sm = c && c->dtype == ZB_F64 ? 2 : 4;
  t.n_classes = 1;
  t.class_max_side[0] = 1 << 30;
  t.edge_rows[0] = SXC_ENS;
  t.interior_rows[0] = SX;
  return t;
}

static bool ens_tuning_valid(const zb_swe2d_cfg* c, const zb_ens_tuning* t) {
  if (!c || !t || (t->tile_x != 8 && t->tile_x != 16)) return false;
  if (t->ctas_per_sm < 1 || t->ctas_per_sm > (c->dtype == ZB_F64 ? 2 : 4)) return false;
  if (t->n_classes < 1 || t->n_classes > 4) return false;
  for (int k = 0; k < t->n_classes; ++k) {
    if (t->edge_rows[k] < 4 || t->edge_rows[k] > SXC_MAX) return false;
    if (t->interior_rows[k] < 8 || t->interior_rows[k] > 1024) return false;
    if (k > 0 && t->class_max_side[k] <= t->class_max_side[k - 1]) return false;
  }
  return true;
}

static bool ens_valid(const zb_swe2d_cfg* c, const zb_ens_instance* inst, int n, int tile_x) {
  if (!c || !inst || n < 1 || (tile_x != 8 && tile_x != 16)) return false;
  if (c->order != 2 || c->recon != ZB_RECON_ETA || c->riemann != ZB_RIEMANN_HLL_HR) return false;
  if (c->dtype != ZB_F32 && c->dtype != ZB_F64) return false;
  for (int i = 0; i < 4; ++i)
    if (c->bc[i] != ZB_BC_WALL && c->bc[i] != ZB_BC_EXTRAPOLATION) return false;
  for (int i = 0; i < n; ++i)
    if (inst[i].nx < 3 || inst[i].ny < 3 || !(inst[i].dx > 0) || !(inst[i].dy > 0) ||
        inst[i].q_offset < 0 || inst[i].ws_offset < 0)
      return false;
  return true;
}

template <typename T, int TX>
static int ens_launch(int part, const void* table, int n_inst, int n_items, int grid,
                      int ctas_per_sm, void* Q, void* W, zb_ctrl* ctrls, int phase,
                      cudaStream_t st) {
  const EnsDesc<T>* desc = (const EnsDesc<T>*)table;
  const int4* items = (const int4*)((const char*)table + ens_desc_bytes<T>(n_inst));
  const size_t sm = sizeof(Smem<T, TX>);
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 32) return ZB_E_UNSUPPORTED;
  static std::atomic<int> sms_cache[32];
  if (!sms_cache[dev].load()) {
    int v = 0;
    ZB_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    sms_cache[dev].store(v);
  }
  // boundary strips, interior strips (persistent warps over their items; a
  // grid that finds none exits at once), then the tiles of grids too small
  // for strips
  const int sgrid_e = sms_cache[dev].load() * ctas_per_sm;
  const int sgrid_i = sgrid_e;
  // the boundary items on the library's second stream, beside the interior ones
  SideStream* side = nullptr;
  {
    const int rc = side_stream(&side);
    if (rc) return rc;
  }
  ZB_CUDA_TRY(cudaEventRecord(side->fork, st));
  ZB_CUDA_TRY(cudaStreamWaitEvent(side->s, side->fork, 0));
  // the column-EDGE items (longer) before the EDGE items on the second stream
  if (part == 0) {
    ens_strip_kernel<T, MODE_STEP1, 3><<<sgrid_e, STRIP_NT, 0, side->s>>>(
        desc, items, (T*)Q, (T*)W, ctrls, phase);
    ens_strip_kernel<T, MODE_STEP1, 1><<<sgrid_e, STRIP_NT, 0, side->s>>>(
        desc, items, (T*)Q, (T*)W, ctrls, phase);
    ens_strip_kernel<T, MODE_STEP1, 0><<<sgrid_i, STRIP_NT, 0, st>>>(desc, items, (T*)Q,
                                                                    (T*)W, ctrls, phase);
  } else {
    ens_strip_kernel<T, MODE_STEP2, 3><<<sgrid_e, STRIP_NT, 0, side->s>>>(
        desc, items, (T*)Q, (T*)W, ctrls, phase);
    ens_strip_kernel<T, MODE_STEP2, 1><<<sgrid_e, STRIP_NT, 0, side->s>>>(
        desc, items, (T*)Q, (T*)W, ctrls, phase);
    ens_strip_kernel<T, MODE_STEP2, 0><<<sgrid_i, STRIP_NT, 0, st>>>(desc, items, (T*)Q,
                                                                    (T*)W, ctrls, phase);
  }
  ZB_CUDA_TRY(cudaGetLastError());
  ZB_CUDA_TRY(cudaEventRecord(side->join, side->s));
  ZB_CUDA_TRY(cudaStreamWaitEvent(st, side->join, 0));
  // the tile fallback (grids narrower than four cells; its CTAs exit at once
  // when the work list holds no tile items)
  static std::atomic<unsigned> mask1{0u};
  auto k1 = ens_stage_kernel<T, TX, 2, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR, MODE_STEP1>;
  auto k2 = ens_stage_kernel<T, TX, 2, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR, MODE_STEP2>;
  if (!(mask1.load() & (1u << dev))) {
    ZB_CUDA_TRY(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    ZB_CUDA_TRY(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    mask1.fetch_or(1u << dev);
  }
  if (grid <= 0) {
    int per_sm = 0, sms = 0;
    ZB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k1, NT, sm));
    ZB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    grid = std::max(1, per_sm) * sms;
  }
  grid = std::min(grid, n_items);
  if (part == 0)
    k1<<<grid, NT, sm, st>>>(desc, items, (T*)Q, (T*)W, ctrls, phase);
  else
    k2<<<grid, NT, sm, st>>>(desc, items, (T*)Q, (T*)W, ctrls, phase);
  return zb_launch_check();
}

}  // namespace zb

using namespace zb;

extern "C" {

const char* zb_version(void) { return "libzb 0.1 (sm_100a)"; }

size_t zb_swe2d_workspace_bytes(const zb_swe2d_cfg* cfg) {
  if (!valid_cfg(cfg)) return 0;
  const size_t es = cfg->dtype == ZB_F64 ? 8 : 4;
  return 3 * (size_t)cfg->nx * cfg->ny * es + 256;
}

size_t zb_swe2d_bed_bytes(const zb_swe2d_cfg* cfg) {
  if (!valid_cfg(cfg) || !bed_scheme(cfg)) return 0;
  return 3 * (size_t)cfg->nx * cfg->ny * (cfg->dtype == ZB_F64 ? 8 : 4);
}

int zb_swe2d_bed_prepare(const zb_swe2d_cfg* cfg, const void* Q, void* bed, size_t bed_bytes,
                         zb_stream_t stream) {
  if (!valid_cfg(cfg) || !bed_scheme(cfg) || !Q || !bed) return ZB_E_ARG;
  if (bed_bytes < zb_swe2d_bed_bytes(cfg) || ((uintptr_t)bed & 7u)) return ZB_E_ARG;
  const size_t n = (size_t)cfg->nx * cfg->ny;
  const int grid = (int)std::min<size_t>((n + NT - 1) / NT, (size_t)148 * 16);
  if (cfg->dtype == ZB_F64) {
    const SweParams<double> p = make_params<double>(cfg, 0.0, 1.0);
    swe2d_bed_kernel<double><<<grid, NT, 0, (cudaStream_t)stream>>>((const double*)Q,
                                                                     (double*)bed, p);
  } else {
    const SweParams<float> p = make_params<float>(cfg, 0.0, 1.0);
    swe2d_bed_kernel<float><<<grid, NT, 0, (cudaStream_t)stream>>>((const float*)Q,
                                                                   (float*)bed, p);
  }
  return zb_launch_check();
}

int zb_swe2d_init(const zb_swe2d_cfg* cfg, const void* Q, zb_ctrl* ctrl, int phase,
                  double t0, zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !ctrl || phase < 0 || phase > 2) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  {
    // the second stream of the fused step is created here, outside any capture
    SideStream* side = nullptr;
    const int rc = side_stream(&side);
    if (rc) return rc;
  }
  swe2d_ctrl_init_kernel<<<1, 32, 0, st>>>(ctrl, phase, t0);
  if (cfg->dtype == ZB_F32) return amax_into<float>(cfg, (const float*)Q, &ctrl->amax[phase], st);
  return amax_into<double>(cfg, (const double*)Q, &ctrl->amax[phase], st);
}

int zb_swe2d_dt(const zb_swe2d_cfg* cfg, const void* Q, zb_ctrl* ctrl, double t,
                zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !ctrl) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  int rc = cfg->dtype == ZB_F32
               ? amax_into<float>(cfg, (const float*)Q, &ctrl->reserved[0], st)
               : amax_into<double>(cfg, (const double*)Q, &ctrl->reserved[0], st);
  if (rc) return rc;
  const double r_in = cfg->dx * cfg->dy / (cfg->dx + cfg->dy);
  swe2d_dt_finalize_kernel<<<1, 32, 0, st>>>(
      ctrl, t, cfg->cfl * 2.0 * r_in,
      (double)cfg->dim_factor * (double)(2 * cfg->degree + 1), cfg->dt_max, cfg->t_end);
  return zb_launch_check();
}

int zb_swe2d_step_part(const zb_swe2d_cfg* cfg, void* Q, void* workspace,
                       size_t workspace_bytes, zb_ctrl* ctrl, int phase, int part,
                       zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !ctrl || phase < 0 || phase > 2) return ZB_E_ARG;
  if (part < -1 || part > 1) return ZB_E_ARG;
  if (!workspace || workspace_bytes < zb_swe2d_workspace_bytes(cfg)) return ZB_E_ARG;
  if (cfg->recon == ZB_RECON_ETA && cfg->riemann == ZB_RIEMANN_RUSANOV) return ZB_E_UNSUPPORTED;
  cudaStream_t st = (cudaStream_t)stream;
  if (cfg->dtype == ZB_F32) {
    return dispatch<float>(cfg, [&](auto O, auto R, auto M) {
      return run_step<float, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
          cfg, (float*)Q, (float*)workspace, ctrl, phase, part, st);
    });
  }
  return dispatch<double>(cfg, [&](auto O, auto R, auto M) {
    return run_step<double, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
        cfg, (double*)Q, (double*)workspace, ctrl, phase, part, st);
  });
}

int zb_swe2d_step(const zb_swe2d_cfg* cfg, void* Q, void* workspace, size_t workspace_bytes,
                  zb_ctrl* ctrl, int phase, zb_stream_t stream) {
  return zb_swe2d_step_part(cfg, Q, workspace, workspace_bytes, ctrl, phase, -1, stream);
}

int zb_swe2d_stage(const zb_swe2d_cfg* cfg, const void* Qk, const void* Q0, void* Q_out,
                   double alpha, double beta, double dt, const void* hinv_src,
                   const uint8_t* force_o1, uint8_t* trouble_out, zb_ctrl* ctrl,
                   zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Qk || !Q_out || !ctrl) return ZB_E_ARG;
  if (Q_out == Qk) return ZB_E_ARG;
  if (!(dt >= 0.0) && !(dt < 0.0)) return ZB_E_ARG;
  if (alpha != 0.0 && !Q0) return ZB_E_ARG;
  if (cfg->recon == ZB_RECON_ETA && cfg->riemann == ZB_RIEMANN_RUSANOV) return ZB_E_UNSUPPORTED;
  cudaStream_t st = (cudaStream_t)stream;
  if (cfg->dtype == ZB_F32) {
    return dispatch<float>(cfg, [&](auto O, auto R, auto M) {
      return run_generic_stage<float, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
          cfg, (const float*)Qk, (const float*)Q0, (float*)Q_out, alpha, beta, dt, ctrl,
          (const float*)hinv_src, force_o1, trouble_out, st);
    });
  }
  return dispatch<double>(cfg, [&](auto O, auto R, auto M) {
    return run_generic_stage<double, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
        cfg, (const double*)Qk, (const double*)Q0, (double*)Q_out, alpha, beta, dt, ctrl,
        (const double*)hinv_src, force_o1, trouble_out, st);
  });
}

int zb_swe2d_source(const zb_swe2d_cfg* cfg, void* Q, const void* hinv0, double dt,
                    zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !hinv0 || !(dt >= 0.0)) return ZB_E_ARG;
  if (cfg->manning_n == 0.0) return ZB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t C = (size_t)cfg->nx * cfg->ny;
  const int blocks = (int)std::min<size_t>((C + NT - 1) / NT, 148 * 16);
  if (cfg->dtype == ZB_F32)
    swe2d_source_kernel<float><<<blocks, NT, 0, st>>>(
        (float*)Q + 2 * C, (float*)Q + 3 * C, (const float*)hinv0, C, (float)cfg->g,
        (float)cfg->manning_n, (float)dt, cfg->implicit_source);
  else
    swe2d_source_kernel<double><<<blocks, NT, 0, st>>>(
        (double*)Q + 2 * C, (double*)Q + 3 * C, (const double*)hinv0, C, cfg->g,
        cfg->manning_n, dt, cfg->implicit_source);
  return zb_launch_check();
}

size_t zb_swe2d_mass_partials(const zb_swe2d_cfg* cfg) {
  (void)cfg;
  return MASS_BLOCKS;
}

int zb_swe2d_mass(const zb_swe2d_cfg* cfg, const void* Q, double* partial, zb_ctrl* ctrl,
                  zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !partial || !ctrl) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t C = (size_t)cfg->nx * cfg->ny;
  const double vol = cfg->dx * cfg->dy;
  if (cfg->dtype == ZB_F32)
    mass_partial_kernel<float><<<MASS_BLOCKS, NT, 0, st>>>((const float*)Q + C, C, vol, partial);
  else
    mass_partial_kernel<double><<<MASS_BLOCKS, NT, 0, st>>>((const double*)Q + C, C, vol, partial);
  mass_final_kernel<<<1, NT, 0, st>>>(partial, MASS_BLOCKS, ctrl);
  return zb_launch_check();
}

int zb_swe2d_aux(const zb_swe2d_cfg* cfg, const void* Q, void* Qaux, zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !Qaux) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t C = (size_t)cfg->nx * cfg->ny;
  const int blocks = (int)std::min<size_t>((C + NT - 1) / NT, 148 * 16);
  if (cfg->dtype == ZB_F32)
    swe2d_aux_kernel<float><<<blocks, NT, 0, st>>>((const float*)Q, (float*)Qaux, cfg->nx,
                                                   cfg->ny, (float)cfg->wet_dry_eps,
                                                   make_lsq<float>(cfg->dx, cfg->dy));
  else
    swe2d_aux_kernel<double><<<blocks, NT, 0, st>>>((const double*)Q, (double*)Qaux, cfg->nx,
                                                    cfg->ny, cfg->wet_dry_eps,
                                                    make_lsq<double>(cfg->dx, cfg->dy));
  return zb_launch_check();
}

int zb_newton_check_f64(const double* a, const double* b, double* out, int64_t n,
                        zb_stream_t stream) {
  if (!a || !b || !out || n < 0) return ZB_E_ARG;
  if (n == 0) return ZB_OK;
  const int blocks = (int)std::min<long long>((n + NT - 1) / NT, 148 * 8);
  newton_check_kernel<<<blocks, NT, 0, (cudaStream_t)stream>>>(a, b, out, (long long)n);
  return zb_launch_check();
}

// ── allocation-free step ────────────────────────────────────────────────────
// Some callers cannot call cudaMalloc: a framework that owns every device
// byte hands a plugin only its operands (an XLA / JAX FFI custom call
// declared without a scratch buffer, an inference-engine plugin at enqueue
// time), and the plugin has no way to ask for more.  For them the stage-1
// state of the fused step lives in this file-scope device array instead of a
// caller workspace: three planes of up to ZB_NOALLOC_MAX_CELLS cells in
// float64 (float32 uses the first half), 24 MiB plus 256 bytes of padding.
// Every GPU that loads libzb holds the array until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[3 * ZB_NOALLOC_MAX_CELLS + 32];

// The array's name in host code is only a host-side stand-in; the kernels
// need its device address, fetched once per device with that device current.
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64] = {};

static int noalloc_scratch(void** out) {
  int dev = -1;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return ZB_E_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return ZB_E_CUDA;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return ZB_OK;
}

int zb_swe2d_step_noalloc(const zb_swe2d_cfg* cfg, void* Q, zb_ctrl* ctrl, int phase,
                          zb_stream_t stream) {
  if (!valid_cfg(cfg) || !Q || !ctrl || phase < 0 || phase > 2) return ZB_E_ARG;
  if ((size_t)cfg->nx * (size_t)cfg->ny > (size_t)ZB_NOALLOC_MAX_CELLS) return ZB_E_TOO_LARGE;
  void* ws = nullptr;
  const int rc = noalloc_scratch(&ws);
  if (rc != ZB_OK) return rc;
  return zb_swe2d_step(cfg, Q, ws, sizeof(g_noalloc_scratch), ctrl, phase, stream);
}


// ── ensemble C ABI ──────────────────────────────────────────────────────────
size_t zb_ens_table_bytes_tuned(const zb_swe2d_cfg* common, const zb_ens_instance* inst,
                                int n_inst, const zb_ens_tuning* tuning) {
  if (!ens_tuning_valid(common, tuning)) return 0;
  if (!ens_valid(common, inst, n_inst, tuning->tile_x)) return 0;
  size_t tiles = 0, strips = 0;
  ens_counts(inst, n_inst, *tuning, &tiles, &strips);
  const size_t d = common->dtype == ZB_F64 ? ens_desc_bytes<double>(n_inst)
                                           : ens_desc_bytes<float>(n_inst);
  return d + (1 + tiles + strips) * sizeof(int4);
}

size_t zb_ens_table_bytes(const zb_swe2d_cfg* common, const zb_ens_instance* inst, int n_inst,
                          int tile_x) {
  if (!common) return 0;
  const zb_ens_tuning t = ens_default_tuning(common, tile_x);
  return zb_ens_table_bytes_tuned(common, inst, n_inst, &t);
}

int zb_ens_prepare(const zb_swe2d_cfg* common, const zb_ens_instance* inst, int n_inst,
                   int tile_x, void* table, size_t table_bytes, int* n_items_out) {
  if (!common) return ZB_E_ARG;
  const zb_ens_tuning t = ens_default_tuning(common, tile_x);
  return zb_ens_prepare_tuned(common, inst, n_inst, &t, table, table_bytes, n_items_out);
}

int zb_ens_prepare_tuned(const zb_swe2d_cfg* common, const zb_ens_instance* inst, int n_inst,
                         const zb_ens_tuning* tuning, void* table, size_t table_bytes,
                         int* n_items_out) {
  if (!ens_tuning_valid(common, tuning)) return ZB_E_ARG;
  const int tile_x = tuning->tile_x;
  if (!ens_valid(common, inst, n_inst, tile_x) || !table || !n_items_out) return ZB_E_ARG;
  if (table_bytes < zb_ens_table_bytes_tuned(common, inst, n_inst, tuning)) return ZB_E_ARG;
  auto build = [&](auto tag) -> int {
    using T = decltype(tag);
    std::vector<EnsDesc<T>> desc(n_inst);
    // items[0]: {tile items, interior strip items, EDGE strip items,
    // column-EDGE strip items}
    std::vector<int4> items(1), strips, estrips, cstrips;
    for (int i = 0; i < n_inst; ++i) {
      zb_swe2d_cfg c = *common;
      c.bed = nullptr;   // instances read their own b; no prepared bed planes
      c.nx = inst[i].nx;
      c.ny = inst[i].ny;
      c.dx = inst[i].dx;
      c.dy = inst[i].dy;
      c.manning_n = inst[i].manning_n;
      c.t_end = inst[i].t_end;
      std::memset(&desc[i], 0, sizeof(EnsDesc<T>));
      desc[i].p = make_params<T>(&c, 0.0, 1.0);
      desc[i].q_off = inst[i].q_offset;
      desc[i].ws_off = inst[i].ws_offset;
      const Fast f = fast_region(c.nx, c.ny);
      desc[i].p.fast_i0 = f.i0; desc[i].p.fast_i1 = f.i1;
      desc[i].p.fast_j0 = f.j0; desc[i].p.fast_j1 = f.j1;
      desc[i].p.strip_full = f.nstrips > 0 ? 1 : 0;
      // tile (0, 0) or strip item (0, 0) keeps the lead duties
      ens_frame_tiles(inst[i], tile_x, [&](int i0, int j0) {
        items.push_back(make_int4(i, i0, j0, i0 == 0 && j0 == 0));
      });
      ens_strip_items(inst[i], *tuning, [&](int st, int r0, int r1, int fl) {
        std::vector<int4>& to = (fl & 4) ? cstrips : ((fl & 1) ? estrips : strips);
        to.push_back(make_int4(i, st, r0, fl | (r1 << 3)));
      });
    }
    // longest items first: the persistent warps take items round-robin, so
    // each warp's k-th item is about as long as every other warp's k-th
    auto longest_first = [](std::vector<int4>& v) {
      std::stable_sort(v.begin(), v.end(), [](const int4& a, const int4& b) {
        return (a.w >> 3) - a.z > (b.w >> 3) - b.z;
      });
    };
    longest_first(strips);
    longest_first(estrips);
    longest_first(cstrips);
    items[0] = make_int4((int)(items.size() - 1), (int)strips.size(), (int)estrips.size(),
                         (int)cstrips.size());
    items.insert(items.end(), strips.begin(), strips.end());
    items.insert(items.end(), estrips.begin(), estrips.end());
    items.insert(items.end(), cstrips.begin(), cstrips.end());
    const size_t db = ens_desc_bytes<T>(n_inst);
    // the table may still be read by steps in flight on any stream: wait for
    // the device, copy, and return only once the copy has landed
    ZB_CUDA_TRY(cudaDeviceSynchronize());
    ZB_CUDA_TRY(cudaMemcpy(table, desc.data(), desc.size() * sizeof(EnsDesc<T>),
                           cudaMemcpyHostToDevice));
    ZB_CUDA_TRY(cudaMemcpy((char*)table + db, items.data(), items.size() * sizeof(int4),
                           cudaMemcpyHostToDevice));
    ZB_CUDA_TRY(cudaDeviceSynchronize());
    *n_items_out = (int)items.size() - 1;
    return ZB_OK;
  };
  return common->dtype == ZB_F64 ? build(double()) : build(float());
}

int zb_ens_init(const zb_swe2d_cfg* common, const void* table, int n_inst, const void* Q,
                zb_ctrl* ctrls, int phase, double t0, zb_stream_t stream) {
  if (!common || !table || !Q || !ctrls || n_inst < 1 || phase < 0 || phase > 2) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  {
    SideStream* side = nullptr;   // created here, outside any capture
    const int rc = side_stream(&side);
    if (rc) return rc;
  }
  const int grid = std::min(n_inst, 148 * 8);
  if (common->dtype == ZB_F64)
    ens_amax_kernel<double><<<grid, NT, 0, st>>>((const EnsDesc<double>*)table, (const double*)Q,
                                                 ctrls, n_inst, phase, t0, common->g,
                                                 common->wet_dry_eps);
  else
    ens_amax_kernel<float><<<grid, NT, 0, st>>>((const EnsDesc<float>*)table, (const float*)Q,
                                                ctrls, n_inst, phase, t0, (float)common->g,
                                                (float)common->wet_dry_eps);
  return zb_launch_check();
}

int zb_ens_step_part_tuned(const zb_swe2d_cfg* common, const void* table, int n_inst,
                           int n_items, const zb_ens_tuning* tuning, int grid, void* Q, void* W,
                           zb_ctrl* ctrls, int phase, int part, zb_stream_t stream) {
  if (!common || !table || !Q || !W || !ctrls || n_inst < 1 || n_items < 1) return ZB_E_ARG;
  if (phase < 0 || phase > 2 || part < -1 || part > 1) return ZB_E_ARG;
  if (!ens_tuning_valid(common, tuning)) return ZB_E_ARG;
  const int tile_x = tuning->tile_x, cps = tuning->ctas_per_sm;
  cudaStream_t st = (cudaStream_t)stream;
  for (int pt = (part == 1 ? 1 : 0); pt <= (part == 0 ? 0 : 1); ++pt) {
    int rc;
    if (common->dtype == ZB_F64)
      rc = tile_x == 8
               ? ens_launch<double, 8>(pt, table, n_inst, n_items, grid, cps, Q, W, ctrls, phase, st)
               : ens_launch<double, 16>(pt, table, n_inst, n_items, grid, cps, Q, W, ctrls, phase, st);
    else
      rc = tile_x == 8
               ? ens_launch<float, 8>(pt, table, n_inst, n_items, grid, cps, Q, W, ctrls, phase, st)
               : ens_launch<float, 16>(pt, table, n_inst, n_items, grid, cps, Q, W, ctrls, phase, st);
    if (rc) return rc;
  }
  return ZB_OK;
}

int zb_ens_step_part(const zb_swe2d_cfg* common, const void* table, int n_inst, int n_items,
                     int tile_x, int grid, void* Q, void* W, zb_ctrl* ctrls, int phase,
                     int part, zb_stream_t stream) {
  if (!common || (tile_x != 8 && tile_x != 16)) return ZB_E_ARG;
  const zb_ens_tuning t = ens_default_tuning(common, tile_x);
  return zb_ens_step_part_tuned(common, table, n_inst, n_items, &t, grid, Q, W, ctrls, phase,
                                part, stream);
}

}  // extern "C"
