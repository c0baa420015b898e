// Unstructured-triangle 2-D shallow-water step for sm_100a.
//
// Three launches per stage (zoomy_jax/fvm/solver_jax.py:722-895;
// solver2/blocks.py:129-287, march.py:126-157):
//   tri_grad_kernel   one thread per cell: W = (b, eta, u, v) or (b, h, qx, qy),
//                     least-squares gradient over the three face neighbours /
//                     boundary ghosts, Barth-Jespersen (= the reference's
//                     "minmod") limiter, eta tie and dry demotion -> limited
//                     slopes (8 planes).
//   tri_face_kernel   one thread per face, every face evaluated once: traces
//                     of both sides with the Audusse clip, hydrostatic-
//                     reconstruction HLL / Rusanov, the cell-edge bed term;
//                     writes the owner's and the neighbour's contribution
//                     (6 planes over faces).  On the first stage it also
//                     reduces the CFL dt over faces in float64.
//   tri_update_kernel one thread per cell: gathers its three faces in a fixed
//                     order (deterministic, no atomics, exactly conservative
//                     because each face contributes +F and -F once) and
//                     applies the Shu-Osher update; the last stage adds
//                     Manning friction and the troubled-cell flag.
// Connectivity is int32 (C, F < 2^31); geometry SoA in the state precision.
#include <cstring>
#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace zb {
namespace tri {

constexpr int NT = 256;
enum { MODE_STEP1 = 0, MODE_STEP2 = 1, MODE_EULER = 2, MODE_STAGE = 3 };

template <typename T>
struct Geo {
  // cells
  const int* lsq_idx;   // [3][C]: neighbour cell or -1 - bf
  const T* lsq_wx;      // [3][C]
  const T* lsq_wy;
  const T* cf_rx;       // [3][C]: face centre - cell centre of the slot's face
  const T* cf_ry;
  const int* cell_face; // [3][C]: 2 f + side (0 owner, 1 neighbour)
  const T* cell_inv_area;
  // faces
  const int* face_a;
  const int* face_b;    // >= 0 neighbour, else -1 - bf
  const T* face_nx;
  const T* face_ny;
  const T* face_len;
  const T* face_rax;
  const T* face_ray;
  const T* face_rbx;
  const T* face_rby;
  const double* face_inr;
  // boundary faces
  const int* bf_kind;
  const T* bf_nx;
  const T* bf_ny;
  int C, F, nbf;
};

template <typename T>
struct Prm {
  T g, eps_kp, eps_wet, manning_n;
  int limiter, implicit_source;
  double cfl2, den_fac, dt_max, t_end;
  double alpha, beta, dt_stage;
};

template <typename T, int RECON>
__device__ __forceinline__ void to_w(T b, T h, T qx, T qy, T eps, T w[4], T& hinv) {
  hinv = kp_hinv(h, eps);
  w[0] = b;
  if (RECON == ZB_RECON_ETA) {
    w[1] = b + h;
    w[2] = qx * hinv;
    w[3] = qy * hinv;
  } else {
    w[1] = h;
    w[2] = qx;
    w[3] = qy;
  }
}

// ── gradient + limiter ──────────────────────────────────────────────────────
template <typename T, int RECON>
__global__ void __launch_bounds__(NT)
tri_grad_kernel(const T* __restrict__ Q, T* __restrict__ S, const Geo<T> geo,
                const Prm<T> p, const unsigned char* __restrict__ force_o1) {
  const int C = geo.C;
  const int c = blockIdx.x * NT + threadIdx.x;
  if (c >= C) return;
  const size_t Cs = (size_t)C;
  const T bc_ = Q[c], hc = Q[Cs + c], qxc = Q[2 * Cs + c], qyc = Q[3 * Cs + c];
  T wc[4], hic;
  to_w<T, RECON>(bc_, hc, qxc, qyc, p.eps_kp, wc, hic);
  T d[3][4], gx[4], gy[4], umax[4], umin[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) { gx[v] = T(0); gy[v] = T(0); umax[v] = wc[v]; umin[v] = wc[v]; }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int idx = geo.lsq_idx[k * Cs + c];
    T wn[4];
    T gb[4];   // value entering the bounds
    if (idx >= 0) {
      T hin;
      to_w<T, RECON>(Q[idx], Q[Cs + idx], Q[2 * Cs + idx], Q[3 * Cs + idx], p.eps_kp, wn, hin);
#pragma unroll
      for (int v = 0; v < 4; ++v) gb[v] = wn[v];
    } else {
      // boundary ghost: BC at the cell state (solver2/blocks.py:129-157); a
      // wall mirrors the normal momentum q - 2 (q.n) n
      const int bf = -1 - idx;
      const int kind = geo.bf_kind[bf];
      T gqx = qxc, gqy = qyc;
      if (kind == ZB_BC_WALL) {
        const T nx = geo.bf_nx[bf], ny = geo.bf_ny[bf];
        const T qn = qxc * nx + qyc * ny;
        gqx = qxc - T(2) * qn * nx;
        gqy = qyc - T(2) * qn * ny;
      }
      T hg;
      to_w<T, RECON>(bc_, hc, gqx, gqy, p.eps_kp, wn, hg);
      // bounds see the ghost at 2 u_bf - u (reconstruction_jax.py:535-579)
#pragma unroll
      for (int v = 0; v < 4; ++v) gb[v] = T(2) * wn[v] - wc[v];
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      d[k][v] = wn[v] - wc[v];
      umax[v] = fmx(umax[v], gb[v]);
      umin[v] = fmn(umin[v], gb[v]);
    }
  }
  // gradient: weights are zero for a ghost not counted in a direction
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const T wx = geo.lsq_wx[k * Cs + c], wy = geo.lsq_wy[k * Cs + c];
#pragma unroll
    for (int v = 0; v < 4; ++v) { gx[v] += wx * d[k][v]; gy[v] += wy * d[k][v]; }
  }
  T rx[3], ry[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) { rx[k] = geo.cf_rx[k * Cs + c]; ry[k] = geo.cf_ry[k * Cs + c]; }
  T phi[4];
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    // Barth-Jespersen / clip-min: min over faces of clip(dpos / delta) for
    // delta > eps and clip(dneg / delta) for delta < -eps; the minimum of the
    // positive-side ratios is dpos / max(delta), of the negative side
    // -dneg / max(-delta) (IEEE division is monotone)
    const T dpos = umax[v] - wc[v], dneg = umin[v] - wc[v];
    T mpos = T(0), mneg = T(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T del = gx[v] * rx[k] + gy[v] * ry[k];
      mpos = fmx(mpos, del);
      mneg = fmx(mneg, -del);
    }
    T ph = T(1);
    if (p.limiter != ZB_LIM_NONE) {
      if (mpos > T(1e-30)) ph = fmn(ph, clip01(dpos / mpos));
      if (mneg > T(1e-30)) ph = fmn(ph, clip01(-dneg / mneg));
    }
    phi[v] = ph;
  }
  if (RECON == ZB_RECON_ETA) {
    if (p.eps_wet >= T(0) && hc < p.eps_wet) phi[0] = phi[1] = phi[2] = phi[3] = T(0);
    phi[0] = fmn(phi[0], phi[1]);
    phi[2] = fmn(phi[2], phi[1]);
    phi[3] = fmn(phi[3], phi[1]);
  }
  if (force_o1 != nullptr && force_o1[c]) phi[0] = phi[1] = phi[2] = phi[3] = T(0);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    S[(2 * v) * Cs + c] = phi[v] * gx[v];
    S[(2 * v + 1) * Cs + c] = phi[v] * gy[v];
  }
}

// ── face kernel ─────────────────────────────────────────────────────────────
template <typename T>
struct Side {
  T b, h, qx, qy, ux, uy;
};

template <typename T, int ORDER, int RECON>
__device__ __forceinline__ void face_trace(const T* __restrict__ Q, const T* __restrict__ S,
                                           int c, size_t Cs, T rx, T ry, T eps,
                                           Side<T>& sd, T& hc, T& bcell) {
  const T b = Q[c], h = Q[Cs + c], qx = Q[2 * Cs + c], qy = Q[3 * Cs + c];
  hc = h;
  bcell = b;
  T w[4], hinv;
  to_w<T, RECON>(b, h, qx, qy, eps, w, hinv);
  if (ORDER >= 2) {
#pragma unroll
    for (int v = 0; v < 4; ++v)
      w[v] = w[v] + (S[(2 * v) * Cs + c] * rx + S[(2 * v + 1) * Cs + c] * ry);
  }
  sd.b = w[0];
  if (RECON == ZB_RECON_ETA) {
    const T eta = fmx(w[1], w[0]);
    const T hf = eta - w[0];
    sd.h = hf;
    sd.ux = w[2];
    sd.uy = w[3];
    sd.qx = w[2] * hf;
    sd.qy = w[3] * hf;
  } else {
    sd.h = w[1];
    sd.qx = w[2];
    sd.qy = w[3];
    sd.ux = w[2] * hinv;
    sd.uy = w[3] * hinv;
  }
}

template <typename T, int RIEMANN>
__device__ __forceinline__ void riemann_n(const Side<T>& L, const Side<T>& R, T nx, T ny,
                                          T g, T& Fh, T& Fqx, T& Fqy, T& Dm, T& Dp) {
  const T half = T(0.5);
  const T unL = L.ux * nx + L.uy * ny;
  const T unR = R.ux * nx + R.uy * ny;
  if (RIEMANN == ZB_RIEMANN_RUSANOV) {
    const T cL = sqrt(g * L.h), cR = sqrt(g * R.h);
    const T s = fmx(fabs(unL) + cL, fabs(unR) + cR);
    const T qnL = L.qx * nx + L.qy * ny, qnR = R.qx * nx + R.qy * ny;
    const T pL = half * g * (L.h * L.h), pR = half * g * (R.h * R.h);
    const T hs = half * s;
    Fh = half * (qnL + qnR) - hs * (R.h - L.h);
    Fqx = half * ((L.qx * unL + pL * nx) + (R.qx * unR + pR * nx)) - hs * (R.qx - L.qx);
    Fqy = half * ((L.qy * unL + pL * ny) + (R.qy * unR + pR * ny)) - hs * (R.qy - L.qy);
    Dm = T(0);
    Dp = T(0);
    return;
  }
  const T bs = fmx(L.b, R.b);
  const T hLs = fmx(T(0), L.h + L.b - bs);
  const T hRs = fmx(T(0), R.h + R.b - bs);
  const T cL = sqrt(g * hLs), cR = sqrt(g * hRs);
  const T qLx = hLs * L.ux, qLy = hLs * L.uy, qRx = hRs * R.ux, qRy = hRs * R.uy;
  const T FLh = hLs * unL, FRh = hRs * unR;
  const T pL = half * g * (hLs * hLs), pR = half * g * (hRs * hRs);
  const T FLx = qLx * unL + pL * nx, FLy = qLy * unL + pL * ny;
  const T FRx = qRx * unR + pR * nx, FRy = qRy * unR + pR * ny;
  if (RIEMANN == ZB_RIEMANN_RUSANOV_HR) {
    const T s = fmx(fabs(unL) + cL, fabs(unR) + cR);
    const T hs = half * s;
    Fh = half * (FLh + FRh) - hs * (hRs - hLs);
    Fqx = half * (FLx + FRx) - hs * (qRx - qLx);
    Fqy = half * (FLy + FRy) - hs * (qRy - qLy);
  } else {
    const T SL = fmn(unL - cL, unR - cR), SR = fmx(unL + cL, unR + cR);
    const T sl = fmn(SL, T(0)), sr = fmx(SR, T(0));
    const T den = sr - sl;
    const T inv = den > T(0) ? T(1) / den : T(0);
    const T slsr = sl * sr;
    Fh = (sr * FLh - sl * FRh + slsr * (hRs - hLs)) * inv;
    Fqx = (sr * FLx - sl * FRx + slsr * (qRx - qLx)) * inv;
    Fqy = (sr * FLy - sl * FRy + slsr * (qRy - qLy)) * inv;
  }
  Dm = half * g * (L.h * L.h - hLs * hLs);
  Dp = -(half * g * (R.h * R.h - hRs * hRs));
}

template <typename T, int ORDER, int RECON, int RIEMANN, bool DT>
__global__ void __launch_bounds__(NT)
tri_face_kernel(const T* __restrict__ Q, const T* __restrict__ S, T* __restrict__ Fc,
                const Geo<T> geo, const Prm<T> p, double* dt_slot, unsigned* status) {
  __shared__ double red[NT / 32];
  const int F = geo.F;
  const size_t Cs = (size_t)geo.C, Fs = (size_t)F;
  const int f = blockIdx.x * NT + threadIdx.x;
  double loc = INFINITY;
  if (f < F) {
    const int a = geo.face_a[f], bcode = geo.face_b[f];
    const T nx = geo.face_nx[f], ny = geo.face_ny[f];
    Side<T> A, B;
    T hA, bA, hB, bB;
    face_trace<T, ORDER, RECON>(Q, S, a, Cs, geo.face_rax[f], geo.face_ray[f], p.eps_kp, A, hA, bA);
    if (bcode >= 0) {
      face_trace<T, ORDER, RECON>(Q, S, bcode, Cs, geo.face_rbx[f], geo.face_rby[f], p.eps_kp, B,
                                  hB, bB);
    } else {
      // boundary: Q_R = BC(Q_L) at the reconstructed face state
      // (solver_jax.py:827-858)
      B = A;
      hB = hA;
      bB = bA;
      const int kind = geo.bf_kind[-1 - bcode];
      if (kind == ZB_BC_WALL) {
        const T qn = A.qx * nx + A.qy * ny;
        B.qx = A.qx - T(2) * qn * nx;
        B.qy = A.qy - T(2) * qn * ny;
        const T un = A.ux * nx + A.uy * ny;
        B.ux = A.ux - T(2) * un * nx;
        B.uy = A.uy - T(2) * un * ny;
      }
    }
    T Fh, Fx, Fy, Dm, Dp;
    riemann_n<T, RIEMANN>(A, B, nx, ny, p.g, Fh, Fx, Fy, Dm, Dp);
    T gA = T(0), gB = T(0);
    if (ORDER >= 2) {
      gA = T(0.5) * p.g * (hA + A.h) * (A.b - bA);
      gB = T(0.5) * p.g * (hB + B.h) * (B.b - bB);
    }
    // owner: F + (Dm + gA) n ; neighbour: -F + (Dp - gB) n
    Fc[0 * Fs + f] = Fh;
    Fc[1 * Fs + f] = Fx + (Dm + gA) * nx;
    Fc[2 * Fs + f] = Fy + (Dm + gA) * ny;
    Fc[3 * Fs + f] = -Fh;
    Fc[4 * Fs + f] = -Fx + (Dp - gB) * nx;
    Fc[5 * Fs + f] = -Fy + (Dp - gB) * ny;
    if (DT) {
      // CFL law over faces at the CELL states, owner on both sides of a
      // boundary face (solver2/blocks.py:36-95, context.py:111-117)
      const int bc2 = bcode >= 0 ? bcode : a;
      const T hia = kp_hinv(Q[Cs + a], p.eps_kp), hib = kp_hinv(Q[Cs + bc2], p.eps_kp);
      const T lA = fabs(Q[2 * Cs + a] * hia * nx + Q[3 * Cs + a] * hia * ny) +
                   sqrt(p.g * fmx(Q[Cs + a], T(0)));
      const T lB = fabs(Q[2 * Cs + bc2] * hib * nx + Q[3 * Cs + bc2] * hib * ny) +
                   sqrt(p.g * fmx(Q[Cs + bc2], T(0)));
      const double am = (double)nmax(lA, lB);
      loc = (p.cfl2 * geo.face_inr[f]) / (p.den_fac * am);
      if (loc != loc) loc = -1.0;   // non-finite state: poison the minimum
    }
  }
  if (DT) {
    // block min (non-negative doubles; -1 marks a NaN)
    double v = loc;
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      double w = threadIdx.x < NT / 32 ? red[threadIdx.x] : INFINITY;
      for (int o = 16; o > 0; o >>= 1) w = fmin(w, __shfl_xor_sync(0xffffffffu, w, o));
      if (threadIdx.x == 0) {
        if (w < 0.0) {
          atomicOr(status, (unsigned)ZB_ST_DT_INVALID);
          w = 0.0;
        }
        atomicMin(reinterpret_cast<unsigned long long*>(dt_slot),
                  (unsigned long long)__double_as_longlong(w));
      }
    }
  }
}

// ── cell update ─────────────────────────────────────────────────────────────
template <typename T, int MODE>
__global__ void __launch_bounds__(NT)
tri_update_kernel(const T* __restrict__ Qk, const T* Q0, T* Qo, const T* __restrict__ Fc,
                  const Geo<T> geo, const Prm<T> p, zb_ctrl* ctrl, int phase,
                  const T* __restrict__ hinv_src, unsigned char* __restrict__ trouble_out) {
  const int C = geo.C;
  const size_t Cs = (size_t)C, Fs = (size_t)geo.F;
  const int c = blockIdx.x * NT + threadIdx.x;
  double dtd;
  if (MODE == MODE_STAGE) {
    dtd = p.dt_stage >= 0.0 ? p.dt_stage : ctrl->dt;
  } else {
    const double t = ctrl->t[phase];
    double dt = ctrl->amax[phase];   // min over faces of the local CFL dt
    dt = nmin(dt, p.dt_max);
    dt = nmin(dt, p.t_end - t);
    const bool ok = isfinite(dt) && dt > 0.0 && !(ctrl->status & ZB_ST_DT_INVALID);
    if ((MODE == MODE_STEP1 || MODE == MODE_EULER) && blockIdx.x == 0 && threadIdx.x == 0) {
      if (!ok && t < p.t_end) atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
      ctrl->dt = ok ? dt : 0.0;
      ctrl->t[(phase + 1) % 3] = ok ? t + dt : t;
      ctrl->amax[(phase + 2) % 3] = INFINITY;
    }
    dtd = ok ? dt : 0.0;
  }
  if (c >= C) return;
  const T dtT = T(dtd);
  T dq[3] = {T(0), T(0), T(0)};
  const T ia = geo.cell_inv_area[c];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int code = geo.cell_face[k * Cs + c];
    const int f = code >> 1, side = code & 1;
    const T lw = geo.face_len[f] * ia;
#pragma unroll
    for (int v = 0; v < 3; ++v) dq[v] -= lw * Fc[(3 * side + v) * Fs + f];
  }
  const T hk = Qk[Cs + c], qxk = Qk[2 * Cs + c], qyk = Qk[3 * Cs + c];
  T hn, qxn, qyn;
  if (MODE == MODE_STEP1 || MODE == MODE_EULER) {
    hn = hk + dtT * dq[0];
    qxn = qxk + dtT * dq[1];
    qyn = qyk + dtT * dq[2];
  } else if (MODE == MODE_STEP2) {
    const T h2 = hk + dtT * dq[0], qx2 = qxk + dtT * dq[1], qy2 = qyk + dtT * dq[2];
    hn = T(0.5) * (Q0[Cs + c] + h2);
    qxn = T(0.5) * (Q0[2 * Cs + c] + qx2);
    qyn = T(0.5) * (Q0[3 * Cs + c] + qy2);
  } else {
    const T a = T(p.alpha), bt = T(p.beta);
    T sx = dq[1], sy = dq[2];
    if (hinv_src != nullptr && p.manning_n != T(0)) {
      const T hi = hinv_src[c];
      const T qn = sqrt(qxk * qxk + qyk * qyk);
      const T kf = (-p.g) * (p.manning_n * p.manning_n) * qn * (hi * hi) * cbrt(hi);
      sx += qxk * kf;
      sy += qyk * kf;
    }
    const T h2 = hk + bt * dtT * dq[0], qx2 = qxk + bt * dtT * sx, qy2 = qyk + bt * dtT * sy;
    if (p.alpha != 0.0) {
      hn = a * Q0[Cs + c] + (T(1) - a) * h2;
      qxn = a * Q0[2 * Cs + c] + (T(1) - a) * qx2;
      qyn = a * Q0[3 * Cs + c] + (T(1) - a) * qy2;
    } else {
      hn = h2; qxn = qx2; qyn = qy2;
    }
  }
  if ((MODE == MODE_STEP2 || MODE == MODE_EULER) && p.manning_n != T(0)) {
    const T h0 = (MODE == MODE_STEP2) ? Q0[Cs + c] : hk;
    const T hi0 = kp_hinv(h0, p.eps_kp);
    const T qn = sqrt(qxn * qxn + qyn * qyn);
    const T kf = (-p.g) * (p.manning_n * p.manning_n) * qn * (hi0 * hi0) * cbrt(hi0);
    if (p.implicit_source) {
      const T den = T(1) + dtT * (-kf);
      qxn = qxn / den;
      qyn = qyn / den;
    } else {
      qxn = qxn + dtT * (qxn * kf);
      qyn = qyn + dtT * (qyn * kf);
    }
  }
  Qo[Cs + c] = hn;
  Qo[2 * Cs + c] = qxn;
  Qo[3 * Cs + c] = qyn;
  const bool tr = hn < T(0) || !isfinite(hn) || !isfinite(qxn) || !isfinite(qyn);
  if (trouble_out != nullptr) trouble_out[c] = tr ? 1 : 0;
  if (tr) atomicOr(&ctrl->status, (unsigned)ZB_ST_TROUBLED);
  if ((MODE == MODE_STEP2 || MODE == MODE_EULER) && c == 0 && dtd > 0.0)
    atomicAdd(&ctrl->steps, 1u);
}

__global__ void tri_ctrl_init_kernel(zb_ctrl* ctrl, int phase, double t0) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < 3; ++i) { ctrl->amax[i] = INFINITY; ctrl->t[i] = 0.0; }
    ctrl->t[phase] = t0;
    ctrl->dt = 0.0;
    ctrl->status = 0u;
    ctrl->steps = 0u;
    ctrl->troubled = 0u;
  }
}

__global__ void tri_dt_finalize_kernel(zb_ctrl* ctrl, double t, double dt_max, double t_end) {
  if (threadIdx.x == 0) {
    double dt = ctrl->reserved[0];
    dt = nmin(dt, dt_max);
    dt = nmin(dt, t_end - t);
    ctrl->dt = dt;
    if (!(isfinite(dt) && dt > 0.0) && t < t_end)
      atomicOr(&ctrl->status, (unsigned)ZB_ST_DT_INVALID);
  }
}

__global__ void set_double_kernel(double* p, double v) { *p = v; }

template <typename T>
__global__ void __launch_bounds__(NT)
tri_mass_partial(const T* __restrict__ h, const T* __restrict__ inv_area, size_t C,
                 double* partial) {
  __shared__ double red[NT];
  double acc = 0.0;
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C; k += (size_t)gridDim.x * NT)
    acc += (double)h[k] / (double)inv_area[k];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void tri_mass_final(const double* partial, int n, zb_ctrl* ctrl) {
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

// Manning source RK1 / point-implicit with a given aux plane (ode.py:14-18)
template <typename T>
__global__ void __launch_bounds__(NT)
tri_source_kernel(T* __restrict__ qx, T* __restrict__ qy, const T* __restrict__ hinv0,
                  size_t C, T g, T n, T dt, int implicit) {
  for (size_t k = blockIdx.x * (size_t)NT + threadIdx.x; k < C; k += (size_t)gridDim.x * NT) {
    const T hi0 = hinv0[k];
    T a = qx[k], b = qy[k];
    const T qn = sqrt(a * a + b * b);
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

// post-step aux (solver_jax.py:284-369): LSQ derivative rows with
// extrapolation ghosts (zero delta) and KP hinv, rows
// [dqx/dx, dh/dx, dqy/dy, dh/dy, db/dx, db/dy, hinv]
template <typename T>
__global__ void __launch_bounds__(NT)
tri_aux_kernel(const T* __restrict__ Q, T* __restrict__ A, const Geo<T> geo, T eps) {
  const size_t Cs = (size_t)geo.C;
  const int c = blockIdx.x * NT + threadIdx.x;
  if (c >= geo.C) return;
  T g[4][2] = {{T(0), T(0)}, {T(0), T(0)}, {T(0), T(0)}, {T(0), T(0)}};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int idx = geo.lsq_idx[k * Cs + c];
    if (idx < 0) continue;
    const T wx = geo.lsq_wx[k * Cs + c], wy = geo.lsq_wy[k * Cs + c];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const T d = Q[v * Cs + idx] - Q[v * Cs + c];
      g[v][0] += wx * d;
      g[v][1] += wy * d;
    }
  }
  A[0 * Cs + c] = g[2][0];
  A[1 * Cs + c] = g[1][0];
  A[2 * Cs + c] = g[3][1];
  A[3 * Cs + c] = g[1][1];
  A[4 * Cs + c] = g[0][0];
  A[5 * Cs + c] = g[0][1];
  A[6 * Cs + c] = kp_hinv(Q[Cs + c], eps);
}

// ── host side ───────────────────────────────────────────────────────────────
constexpr int MASS_BLOCKS = 1184;

static bool valid(const zb_tri_cfg* c, const zb_tri_mesh* m) {
  if (!c || !m) return false;
  if (m->n_cells < 1 || m->n_faces < 1 || m->n_bf < 0) return false;
  if (c->order != 1 && c->order != 2) return false;
  if (c->order == 1 && c->recon != ZB_RECON_CONSTANT) return false;
  if (c->order == 2 && c->recon == ZB_RECON_CONSTANT) return false;
  if (c->riemann < 0 || c->riemann > 2) return false;
  if (c->recon == ZB_RECON_ETA && c->riemann == ZB_RIEMANN_RUSANOV) return false;
  if (c->limiter != ZB_LIM_MINMOD && c->limiter != ZB_LIM_BARTH_JESPERSEN &&
      c->limiter != ZB_LIM_NONE)
    return false;
  if (c->dtype != ZB_F32 && c->dtype != ZB_F64) return false;
  const void* req[] = {m->lsq_idx, m->lsq_wx, m->lsq_wy, m->cf_rx, m->cf_ry, m->cell_face,
                       m->cell_inv_area, m->face_a, m->face_b, m->face_nx, m->face_ny,
                       m->face_len, m->face_rax, m->face_ray, m->face_rbx, m->face_rby,
                       m->face_inr};
  for (const void* q : req)
    if (!q) return false;
  if (m->n_bf > 0 && (!m->bf_kind || !m->bf_nx || !m->bf_ny)) return false;
  return true;
}

template <typename T>
static Geo<T> make_geo(const zb_tri_mesh* m) {
  Geo<T> g;
  g.lsq_idx = m->lsq_idx;
  g.lsq_wx = (const T*)m->lsq_wx;
  g.lsq_wy = (const T*)m->lsq_wy;
  g.cf_rx = (const T*)m->cf_rx;
  g.cf_ry = (const T*)m->cf_ry;
  g.cell_face = m->cell_face;
  g.cell_inv_area = (const T*)m->cell_inv_area;
  g.face_a = m->face_a;
  g.face_b = m->face_b;
  g.face_nx = (const T*)m->face_nx;
  g.face_ny = (const T*)m->face_ny;
  g.face_len = (const T*)m->face_len;
  g.face_rax = (const T*)m->face_rax;
  g.face_ray = (const T*)m->face_ray;
  g.face_rbx = (const T*)m->face_rbx;
  g.face_rby = (const T*)m->face_rby;
  g.face_inr = m->face_inr;
  g.bf_kind = m->bf_kind;
  g.bf_nx = (const T*)m->bf_nx;
  g.bf_ny = (const T*)m->bf_ny;
  g.C = m->n_cells;
  g.F = m->n_faces;
  g.nbf = m->n_bf;
  return g;
}

template <typename T>
static Prm<T> make_prm(const zb_tri_cfg* c, double alpha, double beta, double dt_stage) {
  Prm<T> p;
  std::memset(&p, 0, sizeof(p));
  p.g = (T)c->g;
  p.eps_kp = (T)c->wet_dry_eps;
  p.eps_wet = (T)(c->eps_wet < 0 ? -1.0 : c->eps_wet);
  p.manning_n = (T)c->manning_n;
  p.limiter = c->limiter;
  p.implicit_source = c->implicit_source;
  p.cfl2 = c->cfl * 2.0;
  p.den_fac = (double)c->dim_factor * (double)(2 * c->degree + 1);
  p.dt_max = c->dt_max;
  p.t_end = c->t_end;
  p.alpha = alpha;
  p.beta = beta;
  p.dt_stage = dt_stage;
  return p;
}

template <typename T, int ORDER, int RECON, int RIEMANN>
static int stage(const zb_tri_cfg* cfg, const Geo<T>& geo, const Prm<T>& p, const T* Qk,
                 const T* Q0, T* Qo, T* S, T* Fc, zb_ctrl* ctrl, int phase, int mode,
                 const T* hinv_src, const unsigned char* force_o1, unsigned char* trouble,
                 cudaStream_t st) {
  const int gc = (geo.C + NT - 1) / NT, gf = (geo.F + NT - 1) / NT;
  if (ORDER >= 2) tri_grad_kernel<T, RECON><<<gc, NT, 0, st>>>(Qk, S, geo, p, force_o1);
  const bool dt = mode == MODE_STEP1 || mode == MODE_EULER;
  double* slot = &ctrl->amax[phase < 3 ? phase : 0];
  if (dt)
    tri_face_kernel<T, ORDER, RECON, RIEMANN, true>
        <<<gf, NT, 0, st>>>(Qk, S, Fc, geo, p, slot, &ctrl->status);
  else
    tri_face_kernel<T, ORDER, RECON, RIEMANN, false>
        <<<gf, NT, 0, st>>>(Qk, S, Fc, geo, p, slot, &ctrl->status);
  switch (mode) {
    case MODE_STEP1:
      tri_update_kernel<T, MODE_STEP1><<<gc, NT, 0, st>>>(Qk, Q0, Qo, Fc, geo, p, ctrl, phase,
                                                           hinv_src, trouble);
      break;
    case MODE_STEP2:
      tri_update_kernel<T, MODE_STEP2><<<gc, NT, 0, st>>>(Qk, Q0, Qo, Fc, geo, p, ctrl, phase,
                                                           hinv_src, trouble);
      break;
    case MODE_EULER:
      tri_update_kernel<T, MODE_EULER><<<gc, NT, 0, st>>>(Qk, Q0, Qo, Fc, geo, p, ctrl, phase,
                                                           hinv_src, trouble);
      break;
    default:
      tri_update_kernel<T, MODE_STAGE><<<gc, NT, 0, st>>>(Qk, Q0, Qo, Fc, geo, p, ctrl, phase,
                                                           hinv_src, trouble);
  }
  return zb_launch_check();
}

template <typename T, typename Fn>
static int dispatch(const zb_tri_cfg* c, Fn&& f) {
#define ZB_TCASE(O, R, M)                                                        \
  if (c->order == O && c->recon == R && c->riemann == M)                         \
    return f(std::integral_constant<int, O>(), std::integral_constant<int, R>(), \
             std::integral_constant<int, M>());
  ZB_TCASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_RUSANOV)
  ZB_TCASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_RUSANOV_HR)
  ZB_TCASE(1, ZB_RECON_CONSTANT, ZB_RIEMANN_HLL_HR)
  ZB_TCASE(2, ZB_RECON_CONSERVATIVE, ZB_RIEMANN_RUSANOV)
  ZB_TCASE(2, ZB_RECON_CONSERVATIVE, ZB_RIEMANN_HLL_HR)
  ZB_TCASE(2, ZB_RECON_ETA, ZB_RIEMANN_RUSANOV_HR)
  ZB_TCASE(2, ZB_RECON_ETA, ZB_RIEMANN_HLL_HR)
#undef ZB_TCASE
  return ZB_E_UNSUPPORTED;
}

// workspace layout (elements of T): Q1 (4 planes, b unused), slopes (8
// planes over cells), face contributions (6 planes over faces)
template <typename T>
static void ws_split(const zb_tri_mesh* m, void* ws, T** Q1, T** S, T** Fc) {
  T* base = (T*)ws;
  const size_t C = (size_t)m->n_cells, F = (size_t)m->n_faces;
  *Q1 = base;
  *S = base + 4 * C;
  *Fc = base + 12 * C;
  (void)F;
}

template <typename T, int ORDER, int RECON, int RIEMANN>
static int run_step(const zb_tri_cfg* cfg, const zb_tri_mesh* m, T* Q, void* ws,
                    zb_ctrl* ctrl, int phase, cudaStream_t st) {
  const Geo<T> geo = make_geo<T>(m);
  const Prm<T> p = make_prm<T>(cfg, 0.0, 1.0, -1.0);
  T *Q1, *S, *Fc;
  ws_split<T>(m, ws, &Q1, &S, &Fc);
  const size_t C = (size_t)m->n_cells;
  if constexpr (ORDER == 1) {
    int rc = stage<T, ORDER, RECON, RIEMANN>(cfg, geo, p, Q, Q, Q1, S, Fc, ctrl, phase,
                                             MODE_EULER, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    ZB_CUDA_TRY(cudaMemcpyAsync(Q + C, Q1 + C, 3 * C * sizeof(T), cudaMemcpyDeviceToDevice, st));
    return ZB_OK;
  } else {
    // stage 1 reads the b plane of Q through Qk = Q; the stage-1 state Q1
    // holds h, qx, qy in planes 1..3 and Q's b plane is copied once per step
    ZB_CUDA_TRY(cudaMemcpyAsync(Q1, Q, C * sizeof(T), cudaMemcpyDeviceToDevice, st));
    int rc = stage<T, ORDER, RECON, RIEMANN>(cfg, geo, p, Q, Q, Q1, S, Fc, ctrl, phase,
                                             MODE_STEP1, nullptr, nullptr, nullptr, st);
    if (rc) return rc;
    return stage<T, ORDER, RECON, RIEMANN>(cfg, geo, p, Q1, Q, Q, S, Fc, ctrl, phase, MODE_STEP2,
                                           nullptr, nullptr, nullptr, st);
  }
}

}  // namespace tri
}  // namespace zb

using namespace zb;
using namespace zb::tri;

extern "C" {

size_t zb_tri_workspace_bytes(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh) {
  if (!valid(cfg, mesh)) return 0;
  const size_t es = cfg->dtype == ZB_F64 ? 8 : 4;
  return (12 * (size_t)mesh->n_cells + 6 * (size_t)mesh->n_faces) * es + 256;
}

int zb_tri_init(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, zb_ctrl* ctrl, int phase,
                double t0, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !ctrl || phase < 0 || phase > 2) return ZB_E_ARG;
  tri_ctrl_init_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(ctrl, phase, t0);
  return zb_launch_check();
}

int zb_tri_step(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, void* Q, void* workspace,
                size_t workspace_bytes, zb_ctrl* ctrl, int phase, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Q || !ctrl || phase < 0 || phase > 2) return ZB_E_ARG;
  if (!workspace || workspace_bytes < zb_tri_workspace_bytes(cfg, mesh)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  if (cfg->dtype == ZB_F32)
    return tri::dispatch<float>(cfg, [&](auto O, auto R, auto M) {
      return run_step<float, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
          cfg, mesh, (float*)Q, workspace, ctrl, phase, st);
    });
  return tri::dispatch<double>(cfg, [&](auto O, auto R, auto M) {
    return run_step<double, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
        cfg, mesh, (double*)Q, workspace, ctrl, phase, st);
  });
}

int zb_tri_stage(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Qk,
                 const void* Q0, void* Q_out, double alpha, double beta, double dt,
                 const void* hinv_src, const uint8_t* force_o1, uint8_t* trouble_out,
                 void* workspace, size_t workspace_bytes, zb_ctrl* ctrl, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Qk || !Q_out || !ctrl || Q_out == Qk) return ZB_E_ARG;
  if (alpha != 0.0 && !Q0) return ZB_E_ARG;
  if (!workspace || workspace_bytes < zb_tri_workspace_bytes(cfg, mesh)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  auto go = [&](auto tag, auto O, auto R, auto M) {
    using T = decltype(tag);
    const Geo<T> geo = make_geo<T>(mesh);
    const Prm<T> p = make_prm<T>(cfg, alpha, beta, dt);
    T *Q1, *S, *Fc;
    ws_split<T>(mesh, workspace, &Q1, &S, &Fc);
    return stage<T, decltype(O)::value, decltype(R)::value, decltype(M)::value>(
        cfg, geo, p, (const T*)Qk, (const T*)Q0, (T*)Q_out, S, Fc, ctrl, 0, MODE_STAGE,
        (const T*)hinv_src, force_o1, trouble_out, st);
  };
  if (cfg->dtype == ZB_F32)
    return tri::dispatch<float>(cfg, [&](auto O, auto R, auto M) { return go(float(), O, R, M); });
  return tri::dispatch<double>(cfg, [&](auto O, auto R, auto M) { return go(double(), O, R, M); });
}

int zb_tri_dt(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q, void* workspace,
              size_t workspace_bytes, zb_ctrl* ctrl, double t, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Q || !ctrl) return ZB_E_ARG;
  if (!workspace || workspace_bytes < zb_tri_workspace_bytes(cfg, mesh)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  // the first-order face pass carries the CFL reduction; its face results go
  // to the workspace and are discarded.  The minimum lands in reserved[0].
  set_double_kernel<<<1, 1, 0, st>>>(&ctrl->reserved[0], INFINITY);
  auto go = [&](auto tag) {
    using T = decltype(tag);
    const Geo<T> geo = make_geo<T>(mesh);
    Prm<T> p = make_prm<T>(cfg, 0.0, 1.0, -1.0);
    T *Q1, *S, *Fc;
    ws_split<T>(mesh, workspace, &Q1, &S, &Fc);
    const int gf = (geo.F + NT - 1) / NT;
    tri_face_kernel<T, 1, ZB_RECON_CONSTANT, ZB_RIEMANN_RUSANOV_HR, true>
        <<<gf, NT, 0, st>>>((const T*)Q, S, Fc, geo, p, &ctrl->reserved[0], &ctrl->status);
    return zb_launch_check();
  };
  int rc = cfg->dtype == ZB_F32 ? go(float()) : go(double());
  if (rc) return rc;
  tri_dt_finalize_kernel<<<1, 32, 0, st>>>(ctrl, t, cfg->dt_max, cfg->t_end);
  return zb_launch_check();
}

int zb_tri_source(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, void* Q, const void* hinv0,
                  double dt, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Q || !hinv0 || !(dt >= 0.0)) return ZB_E_ARG;
  if (cfg->manning_n == 0.0) return ZB_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t C = (size_t)mesh->n_cells;
  const int blocks = (int)std::min<size_t>((C + NT - 1) / NT, 148 * 16);
  if (cfg->dtype == ZB_F32)
    tri_source_kernel<float><<<blocks, NT, 0, st>>>((float*)Q + 2 * C, (float*)Q + 3 * C,
                                                    (const float*)hinv0, C, (float)cfg->g,
                                                    (float)cfg->manning_n, (float)dt,
                                                    cfg->implicit_source);
  else
    tri_source_kernel<double><<<blocks, NT, 0, st>>>((double*)Q + 2 * C, (double*)Q + 3 * C,
                                                     (const double*)hinv0, C, cfg->g,
                                                     cfg->manning_n, dt, cfg->implicit_source);
  return zb_launch_check();
}

int zb_tri_aux(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q, void* Qaux,
               zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Q || !Qaux) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const int gc = (mesh->n_cells + NT - 1) / NT;
  if (cfg->dtype == ZB_F32)
    tri_aux_kernel<float><<<gc, NT, 0, st>>>((const float*)Q, (float*)Qaux, make_geo<float>(mesh),
                                             (float)cfg->wet_dry_eps);
  else
    tri_aux_kernel<double><<<gc, NT, 0, st>>>((const double*)Q, (double*)Qaux,
                                              make_geo<double>(mesh), cfg->wet_dry_eps);
  return zb_launch_check();
}

size_t zb_tri_mass_partials(void) { return MASS_BLOCKS; }

int zb_tri_mass(const zb_tri_cfg* cfg, const zb_tri_mesh* mesh, const void* Q, double* partial,
                zb_ctrl* ctrl, zb_stream_t stream) {
  if (!valid(cfg, mesh) || !Q || !partial || !ctrl) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t C = (size_t)mesh->n_cells;
  if (cfg->dtype == ZB_F32)
    tri_mass_partial<float><<<MASS_BLOCKS, NT, 0, st>>>((const float*)Q + C,
                                                        (const float*)mesh->cell_inv_area, C,
                                                        partial);
  else
    tri_mass_partial<double><<<MASS_BLOCKS, NT, 0, st>>>((const double*)Q + C,
                                                         (const double*)mesh->cell_inv_area,
                                                         C, partial);
  tri_mass_final<<<1, NT, 0, st>>>(partial, MASS_BLOCKS, ctrl);
  return zb_launch_check();
}

}  // extern "C"
