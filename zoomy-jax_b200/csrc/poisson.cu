// Chorin pressure solve on B200: variable-coefficient Poisson, geometric
// multigrid, flexible CG.
//
// Reference: zoomy_jax/fvm/solver_chorin_vam_jax.py -- chorin_stage (:524-572)
// runs hyperbolic Euler -> pressure solve (_step_pressure_pure :673-883,
// unpreconditioned restarted GMRES on VAM's operator) -> corrector
// (_step_corrector_pure :885-907).  Here the pressure operator is
//   (A p)_i = sum_f c_f (p_i - p_j) / dx^2,   Dirichlet ghost p_j = -p_i,
// c_f the harmonic face mean of c = clip(h, cmin, cmax), the right-hand side
// f = -div(q*) / dt, and the corrector q -= dt * cell-averaged c_f grad p.
//
// Precision: the Krylov vectors, the operator and the residual are float64;
// the multigrid preconditioner runs in float32 (iterative refinement inside
// flexible CG).  Multigrid: cell-centred factor-2 coarsening, coarse face
// coefficient = mean of the two fine faces it covers, bilinear prolongation P
// with odd reflection at the Dirichlet boundary, restriction R = P^T / 4,
// red-black Gauss-Seidel (pre red/black, post black/red), a symmetric V-cycle
// whose coarsest level (at most 64 cells) is solved exactly with an inverse
// built at set-up.  Each level larger than 16 x 16 costs two launches per
// V-cycle: a fused pre-smooth + residual + restriction kernel on the way down
// and a fused prolongation + post-smooth kernel on the way up (32 x 32 tiles
// with a halo in shared memory).  Levels whose side is <= 16 run in ONE CTA
// with every array in shared memory (their launches would otherwise be pure
// latency).  Layout: cell (i, j) at i*ny + j; x-faces (nx+1, ny) at i*ny + j;
// y-faces (nx, ny+1) at i*(ny+1) + j.
#include <cstring>
#include <algorithm>
#include <atomic>
#include <utility>

#include "common.cuh"

namespace zb {
namespace pois {

constexpr int NT = 256;
constexpr int MAXL = 16;
constexpr int SMALL = 32;        // levels with nx, ny <= SMALL go to the one-CTA kernel
constexpr int RED_BLOCKS = 592;  // 148 SMs x 4
constexpr int DENSE_MAX_CELLS = 64;   // coarsest levels this small are solved exactly

struct Level {
  int nx, ny;
  float dx;
  long long cx, cy, idg, x, f, r;   // float offsets into the workspace
  long long xo;                    // the level's V-cycle result (see mg_up_kernel)
};

struct Plan {
  int nlev, small0;          // number of levels, first one-CTA level
  Level L[MAXL];
  long long cx64, cy64, dg64;  // double offsets (level-0 operator)
  long long vr, vp, vq;        // double offsets (Krylov vectors; z is the V-cycle's float32
                               // result on level 0, converted where it is read)
  long long part;              // double offset of the reduction partials
  long long scal;              // double offset of the scalars
  long long cinv;              // float offset of the coarsest inverse (-1: none)
  long long fbase;             // byte offset of the float region
  long long bytes;
  int nu, coarse_sweeps;
  double dx;
};

// Programmatic dependent launch: the kernels of a solve iteration and of the
// V-cycle are launched with programmatic stream serialisation, so the next
// kernel's launch overlaps the tail of this one.  Each of them first waits for
// its predecessor's completion and memory (griddepcontrol.wait, before any
// global read or write), then lets its own successor launch; launched without
// the attribute, both instructions are no-ops.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
static cudaError_t pdl_launch(void (*k)(KArgs...), dim3 g, dim3 b, size_t sm, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t c = {};
  c.gridDim = g;
  c.blockDim = b;
  c.dynamicSmemBytes = sm;
  c.stream = st;
  cudaLaunchAttribute a[1];
  a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  a[0].val.programmaticStreamSerializationAllowed = 1;
  c.attrs = a;
  // only on launches outside stream capture: inside the FCG graph's
  // conditional body the programmatic edges measured slower than plain ones
  // (1024^2 pressure solve, 8 iterations: 1.655 ms against 1.628 ms)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
  c.numAttrs = cs == cudaStreamCaptureStatusNone ? 1 : 0;
  return cudaLaunchKernelEx(&c, k, std::forward<Args>(args)...);
}

// scalars (doubles) at plan.scal
enum { S_BB = 0, S_RR, S_PQ, S_PR, S_ZQ, S_ALPHA, S_BETA, S_REL, S_ITER, S_COUNT = 16 };

static Plan make_plan(const zb_poisson_cfg* c) {
  Plan P;
  std::memset(&P, 0, sizeof(P));
  P.nu = c->nu;
  P.coarse_sweeps = c->coarse_sweeps;
  P.dx = c->dx;
  int nx = c->nx, ny = c->ny;
  float dx = (float)c->dx;
  long long f = 0;
  int l = 0;
  P.small0 = -1;
  // every float array starts on 16 bytes (the fused kernels stage rows with
  // 16-byte copies)
  auto al4 = [](long long v) { return (v + 3) & ~3LL; };
  while (l < MAXL) {
    Level& L = P.L[l];
    L.nx = nx;
    L.ny = ny;
    L.dx = dx;
    L.cx = f; f = al4(f + (long long)(nx + 1) * ny);
    L.cy = f; f = al4(f + (long long)nx * (ny + 1));
    L.idg = f; f = al4(f + (long long)nx * ny);
    L.x = f; f = al4(f + (long long)nx * ny);
    L.f = f; f = al4(f + (long long)nx * ny);
    L.r = f; f = al4(f + (long long)nx * ny);
    L.xo = f; f = al4(f + (long long)nx * ny);
    if (P.small0 < 0 && nx <= SMALL && ny <= SMALL) P.small0 = l;
    ++l;
    if (nx <= c->coarsest || ny <= c->coarsest || (nx & 1) || (ny & 1)) break;
    nx /= 2;
    ny /= 2;
    dx *= 2.0f;
  }
  P.nlev = l;
  if (P.small0 < 0) P.small0 = l;   // no level small enough: no one-CTA part
  {
    const Level& Lc = P.L[l - 1];
    const long long nc = (long long)Lc.nx * Lc.ny;
    if (nc <= DENSE_MAX_CELLS) {
      P.cinv = f;
      f += nc * nc;
    } else {
      P.cinv = -1;
    }
  }
  const long long C = (long long)c->nx * c->ny;
  long long d = 0;
  P.cx64 = d; d += (long long)(c->nx + 1) * c->ny;
  P.cy64 = d; d += (long long)c->nx * (c->ny + 1);
  P.dg64 = d; d += C;
  P.vr = d; d += C;
  P.vp = d; d += C;
  P.vq = d; d += C;
  P.part = d; d += 4 * RED_BLOCKS;
  P.scal = d; d += S_COUNT;
  P.fbase = ((d * 8 + 255) / 256) * 256;
  P.bytes = P.fbase + f * 4 + 256;
  return P;
}

__device__ __forceinline__ double* D(void* ws, long long off) { return (double*)ws + off; }
__device__ __forceinline__ float* F(void* ws, const Plan& P, long long off) {
  return (float*)((char*)ws + P.fbase) + off;
}

// ── set-up kernels ──────────────────────────────────────────────────────────
// Level 0 in one pass over its cells, each coarser level in one pass over its
// cells from the finer level's faces, and the levels of the one-CTA V-cycle
// plus the coarsest inverse in one CTA: every cell evaluates its four faces
// itself (a face shared by two cells is the same expression on the same
// operands, so both get its bits), writes the faces it owns (west and south;
// east and north on the last row and column) and its diagonal.

// face coefficient: the harmonic mean of the two cells' depths clipped to
// [cmin, cmax]; a side outside the grid takes the other cell's alone
template <typename T>
__device__ __forceinline__ double face_coef(const T* h, long long kl, long long kr, bool hasl,
                                            bool hasr, double cmin, double cmax) {
  const double a = hasl ? fmin(fmax((double)h[kl], cmin), cmax) : -1.0;
  const double b = hasr ? fmin(fmax((double)h[kr], cmin), cmax) : -1.0;
  return (a < 0) ? b : (b < 0 ? a : 2.0 * a * b / (a + b));
}

// diagonal of the 5-point operator from a cell's west, east, south and north
// face coefficients (a wall face counts twice: its ghost is -x)
template <typename T>
__device__ __forceinline__ T diag_of(T a, T b, T c, T d, int i, int j, int nx, int ny, T idx2) {
  T s = (a + b) + (c + d);
  if (i == 0) s += a;
  if (i == nx - 1) s += b;
  if (j == 0) s += c;
  if (j == ny - 1) s += d;
  return s * idx2;
}

// level 0: float64 faces and diagonal (the Krylov operator), float32 faces
// and inverse diagonal (the finest multigrid level)
template <typename T>
__global__ void __launch_bounds__(NT)
setup0_kernel(const T* __restrict__ h, int nx, int ny, double cmin, double cmax, double idx2,
              float idx2f, double* __restrict__ cx64, double* __restrict__ cy64,
              double* __restrict__ dg64, float* __restrict__ cx32, float* __restrict__ cy32,
              float* __restrict__ idg32) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    const double w = face_coef(h, k - ny, k, i > 0, true, cmin, cmax);
    const double e = face_coef(h, k, k + ny, true, i + 1 < nx, cmin, cmax);
    const double so = face_coef(h, k - 1, k, j > 0, true, cmin, cmax);
    const double no = face_coef(h, k, k + 1, true, j + 1 < ny, cmin, cmax);
    const long long ky = (long long)i * (ny + 1) + j;
    cx64[k] = w;
    cx32[k] = (float)w;
    cy64[ky] = so;
    cy32[ky] = (float)so;
    if (i == nx - 1) { cx64[k + ny] = e; cx32[k + ny] = (float)e; }
    if (j == ny - 1) { cy64[ky + 1] = no; cy32[ky + 1] = (float)no; }
    dg64[k] = diag_of<double>(w, e, so, no, i, j, nx, ny, idx2);
    idg32[k] = __frcp_rn(
        diag_of<float>((float)w, (float)e, (float)so, (float)no, i, j, nx, ny, idx2f));
  }
}

// coarse cell (I, J): its faces as the means of the two fine faces they
// cover, and its inverse diagonal
__device__ __forceinline__ void coarsen_cell(const float* cxf, const float* cyf, int nxc, int nyc,
                                             float idx2, float* cxc, float* cyc, float* idg,
                                             int I, int J) {
  const int nyf = 2 * nyc;
  const long long fw = (long long)(2 * I) * nyf + 2 * J, fe = fw + 2LL * nyf;
  const long long fs = (long long)(2 * I) * (nyf + 1) + 2 * J, fn = fs + 2;
  const float w = 0.5f * (cxf[fw] + cxf[fw + 1]);
  const float e = 0.5f * (cxf[fe] + cxf[fe + 1]);
  const float so = 0.5f * (cyf[fs] + cyf[fs + (nyf + 1)]);
  const float no = 0.5f * (cyf[fn] + cyf[fn + (nyf + 1)]);
  const long long k = (long long)I * nyc + J, ky = (long long)I * (nyc + 1) + J;
  cxc[k] = w;
  cyc[ky] = so;
  if (I == nxc - 1) cxc[k + nyc] = e;
  if (J == nyc - 1) cyc[ky + 1] = no;
  idg[k] = __frcp_rn(diag_of<float>(w, e, so, no, I, J, nxc, nyc, idx2));
}

__global__ void __launch_bounds__(NT)
coarsen_kernel(const float* __restrict__ cxf, const float* __restrict__ cyf, int nxc, int nyc,
               float idx2, float* __restrict__ cxc, float* __restrict__ cyc,
               float* __restrict__ idg) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nxc * nyc;
       k += (long long)gridDim.x * NT) {
    const int I = (int)(k / nyc), J = (int)(k - (long long)I * nyc);
    coarsen_cell(cxf, cyf, nxc, nyc, idx2, cxc, cyc, idg, I, J);
  }
}

// ── float64 Krylov kernels ──────────────────────────────────────────────────
__device__ __forceinline__ double ghost_or(const double* p, int nx, int ny, int i, int j,
                                           double self) {
  return (i < 0 || i >= nx || j < 0 || j >= ny) ? -self : p[(long long)i * ny + j];
}

__device__ __forceinline__ void block_sum(double v, double* red, double* out) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    double w = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) *out = w;
  }
}

// Grid-wide finish of a two-stage reduction without another launch: every
// block has stored its partial sums; the last block to arrive (a counter in
// the workspace) adds the partials in a fixed order -- the same order and
// arithmetic as a separate reduction kernel, so the result is deterministic --
// derives the FCG scalar and re-arms the counter.  No block waits on another.
enum { FIN_NONE = 0, FIN_REL = 1, FIN_ALPHA = 2, FIN_BETA = 3 };

__device__ void finish_scalars(const double* part_a, const double* part_b, unsigned* counter,
                               double* scal, int dst_a, int dst_b, int what, double* red) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double sa = 0.0, sb = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += NT) {
    sa += __ldcg(part_a + k);
    if (part_b) sb += __ldcg(part_b + k);
  }
  block_sum(sa, red, &scal[dst_a]);
  __syncthreads();
  if (part_b) block_sum(sb, red, &scal[dst_b]);
  __syncthreads();
  if (threadIdx.x == 0) {
    if (what == FIN_REL) {
      scal[S_REL] = sqrt(scal[S_RR] / scal[S_BB]);
    } else if (what == FIN_ALPHA) {
      const double pq = scal[S_PQ];
      scal[S_ALPHA] = pq != 0.0 ? scal[S_PR] / pq : 0.0;
    } else if (what == FIN_BETA) {
      const double pq = scal[S_PQ];
      scal[S_BETA] = pq != 0.0 ? scal[S_ZQ] / pq : 0.0;
    }
    *counter = 0u;
  }
}

// q = A p; partial[b] = sum p.q ; partial2[b] = sum p.r
__global__ void __launch_bounds__(NT)
apply_dot_kernel(const double* __restrict__ cx, const double* __restrict__ cy,
                 const double* __restrict__ p, const double* __restrict__ r,
                 double* __restrict__ q, int nx, int ny, double idx2, double* part_pq,
                 double* part_pr, unsigned* counter, double* scal) {
  pdl_enter();
  __shared__ double red[NT / 32];
  double spq = 0.0, spr = 0.0;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    const double pc = p[k];
    const double v = (cx[(long long)(i + 1) * ny + j] * (pc - ghost_or(p, nx, ny, i + 1, j, pc)) +
                      cx[(long long)i * ny + j] * (pc - ghost_or(p, nx, ny, i - 1, j, pc)) +
                      cy[(long long)i * (ny + 1) + j + 1] * (pc - ghost_or(p, nx, ny, i, j + 1, pc)) +
                      cy[(long long)i * (ny + 1) + j] * (pc - ghost_or(p, nx, ny, i, j - 1, pc))) *
                     idx2;
    if (q) q[k] = v;
    spq += pc * v;
    if (r) spr += pc * r[k];
  }
  block_sum(spq, red, &part_pq[blockIdx.x]);
  __syncthreads();
  if (part_pr) block_sum(spr, red, &part_pr[blockIdx.x]);
  if (counter) finish_scalars(part_pq, part_pr, counter, scal, S_PQ, S_PR, FIN_ALPHA, red);
}

// x += alpha p ; r -= alpha q ; partial r.r ; r32 = (float) r
__global__ void __launch_bounds__(NT)
update_xr_kernel(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                 const double* __restrict__ q, double* scal, long long n,
                 double* part_rr, float* __restrict__ r32, unsigned* counter) {
  pdl_enter();
  __shared__ double red[NT / 32];
  const double a = scal[S_ALPHA];
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT) {
    x[k] += a * p[k];
    const double rk = r[k] - a * q[k];
    r[k] = rk;
    s += rk * rk;
    if (r32) r32[k] = (float)rk;
  }
  block_sum(s, red, &part_rr[blockIdx.x]);
  finish_scalars(part_rr, nullptr, counter, scal, S_RR, 0, FIN_REL, red);
}

// partial z.q with z = (double) z32, the V-cycle's float32 result (the
// conversion is exact, so z is never stored in float64)
__global__ void __launch_bounds__(NT)
zq_kernel(const float* __restrict__ z32, const double* __restrict__ q, long long n,
          double* part_zq, unsigned* counter, double* scal) {
  pdl_enter();
  __shared__ double red[NT / 32];
  double s = 0.0;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT)
    s += (double)z32[k] * q[k];
  block_sum(s, red, &part_zq[blockIdx.x]);
  finish_scalars(part_zq, nullptr, counter, scal, S_ZQ, 0, FIN_BETA, red);
}

// p = z - beta p, z = (double) z32
__global__ void p_update_kernel(double* __restrict__ p, const float* __restrict__ z32,
                                const double* scal, long long n, int first) {
  pdl_enter();
  const double b = first ? 0.0 : scal[S_BETA];
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT)
    p[k] = first ? (double)z32[k] : (double)z32[k] - b * p[k];
}

// loop control of the graph solve: counts the iteration and keeps the WHILE
// node running while the relative residual is above tol (NaN stops it)
__device__ __forceinline__ void fcg_loop_control(double* scal, cudaGraphConditionalHandle h,
                                                 double tol, int maxit, int first) {
  const double it = first ? 0.0 : scal[S_ITER] + 1.0;
  scal[S_ITER] = it;
  const double rel = scal[S_REL];
  const bool go = rel > tol && it < (double)maxit;   // false for NaN
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// p_update with the graph solve's loop control folded in (block 0, thread 0;
// it reads S_REL, set by update_xr before the V-cycle, and writes S_ITER,
// which p_update does not touch): one launch fewer per iteration
__global__ void p_update_cond_kernel(double* __restrict__ p, const float* __restrict__ z32,
                                     double* scal, long long n, int first,
                                     cudaGraphConditionalHandle h, double tol, int maxit) {
  pdl_enter();
  const double b = first ? 0.0 : scal[S_BETA];
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT)
    p[k] = first ? (double)z32[k] : (double)z32[k] - b * p[k];
  if (blockIdx.x == 0 && threadIdx.x == 0) fcg_loop_control(scal, h, tol, maxit, first);
}

// r = b - A x ; partial r.r and b.b ; r32
__global__ void __launch_bounds__(NT)
residual64_kernel(const double* __restrict__ cx, const double* __restrict__ cy,
                  const double* __restrict__ x, const double* __restrict__ b,
                  double* __restrict__ r, int nx, int ny, double idx2, double* part_rr,
                  double* part_bb, float* __restrict__ r32, unsigned* counter, double* scal) {
  pdl_enter();
  __shared__ double red[NT / 32];
  double srr = 0.0, sbb = 0.0;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    const double pc = x[k];
    const double ax = (cx[(long long)(i + 1) * ny + j] * (pc - ghost_or(x, nx, ny, i + 1, j, pc)) +
                       cx[(long long)i * ny + j] * (pc - ghost_or(x, nx, ny, i - 1, j, pc)) +
                       cy[(long long)i * (ny + 1) + j + 1] * (pc - ghost_or(x, nx, ny, i, j + 1, pc)) +
                       cy[(long long)i * (ny + 1) + j] * (pc - ghost_or(x, nx, ny, i, j - 1, pc))) *
                      idx2;
    const double rk = b[k] - ax;
    r[k] = rk;
    srr += rk * rk;
    sbb += b[k] * b[k];
    if (r32) r32[k] = (float)rk;
  }
  block_sum(srr, red, &part_rr[blockIdx.x]);
  __syncthreads();
  block_sum(sbb, red, &part_bb[blockIdx.x]);
  finish_scalars(part_rr, part_bb, counter, scal, S_RR, S_BB, FIN_REL, red);
}

// ── float32 multigrid kernels ───────────────────────────────────────────────
__device__ __forceinline__ float gx(const float* x, int nx, int ny, int i, int j, float self) {
  return (i < 0 || i >= nx || j < 0 || j >= ny) ? -self : x[i * ny + j];
}

__device__ __forceinline__ float apply_at(const float* x, const float* cx, const float* cy,
                                          int nx, int ny, int i, int j, float idx2,
                                          float& offdiag_sum) {
  const float xc = x[i * ny + j];
  const float a = cx[(i + 1) * ny + j], b = cx[i * ny + j];
  const float c = cy[i * (ny + 1) + j + 1], d = cy[i * (ny + 1) + j];
  const float xe = gx(x, nx, ny, i + 1, j, xc), xw = gx(x, nx, ny, i - 1, j, xc);
  const float xn = gx(x, nx, ny, i, j + 1, xc), xs = gx(x, nx, ny, i, j - 1, xc);
  offdiag_sum = (a * xe + b * xw + c * xn + d * xs) * idx2;
  return (a * (xc - xe) + b * (xc - xw) + c * (xc - xn) + d * (xc - xs)) * idx2;
}

// sum of c_f x_j over the in-domain neighbours (a wall's ghost -x_i belongs
// to the diagonal): the red-black update in the form
// x_i = (f_i + idx2 * sum) / d_i, d_i containing the ghost terms
__device__ __forceinline__ float nbsum_at(const float* x, const float* cx, const float* cy,
                                          int nx, int ny, int i, int j) {
  const float a = cx[(i + 1) * ny + j], b = cx[i * ny + j];
  const float c = cy[i * (ny + 1) + j + 1], d = cy[i * (ny + 1) + j];
  const float xe = i + 1 < nx ? x[(i + 1) * ny + j] : 0.0f;
  const float xw = i > 0 ? x[(i - 1) * ny + j] : 0.0f;
  const float xn = j + 1 < ny ? x[i * ny + j + 1] : 0.0f;
  const float xs = j > 0 ? x[i * ny + j - 1] : 0.0f;
  return (a * xe + b * xw) + (c * xn + d * xs);
}

// one red-black half sweep: x_i = (f_i + idx2 sum_j c_ij x_j) / d_i on cells
// of `color` (the same update as x_i += (f_i - (A x)_i) / d_i)
__global__ void __launch_bounds__(NT)
rbgs_kernel(float* __restrict__ x, const float* __restrict__ f, const float* __restrict__ cx,
            const float* __restrict__ cy, const float* __restrict__ idg, int nx, int ny,
            float idx2, int color) {
  const int half = (ny + 1) / 2;
  for (long long t = blockIdx.x * (long long)NT + threadIdx.x; t < (long long)nx * half;
       t += (long long)gridDim.x * NT) {
    const int i = (int)(t / half), m = (int)(t - (long long)i * half);
    const int j = 2 * m + ((i + color) & 1);
    if (j >= ny) continue;
    x[i * ny + j] = (f[i * ny + j] + idx2 * nbsum_at(x, cx, cy, nx, ny, i, j)) * idg[i * ny + j];
  }
}

__global__ void __launch_bounds__(NT)
residual32_kernel(const float* __restrict__ x, const float* __restrict__ f,
                  const float* __restrict__ cx, const float* __restrict__ cy,
                  float* __restrict__ r, int nx, int ny, float idx2) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    float od;
    r[k] = f[k] - apply_at(x, cx, cy, nx, ny, i, j, idx2, od);
  }
}

// One axis of the bilinear cell-centred prolongation with odd reflection at
// the Dirichlet wall: the weight with which fine index fi (of 2 nc) takes
// coarse index I.  A fine cell takes 3/4 of its own coarse cell and 1/4 of the
// neighbour on its side; a neighbour beyond the wall is the reflection -e of
// the own cell.  The 2-D weights are products of the two axes (9, 3, 3, 1)/16.
__device__ __forceinline__ float w1d(int fi, int I, int nc) {
  const int ci = fi >> 1, nb = ci + ((fi & 1) ? 1 : -1);
  float w = 0.0f;
  if (ci == I) w += 0.75f;
  if (nb == I) w += 0.25f;
  if ((nb < 0 || nb >= nc) && ci == I) w -= 0.25f;
  return w;
}

// restriction R = P^T / 4 at coarse cell (I, J) of a fine residual read by
// rf(fi, fj) (fine indices in range); the fixed loop order makes every
// implementation below produce the same bits
template <typename F>
__device__ __forceinline__ float restrict_at(F rf, int I, int J, int nxc, int nyc) {
  if (I >= 1 && I <= nxc - 2 && J >= 1 && J <= nyc - 2) {
    // away from the wall every fine index is in range and the weights are
    // w1d's constants (1/4, 3/4, 3/4, 1/4): the same sums in the same order
    const float w[4] = {0.25f, 0.75f, 0.75f, 0.25f};
    float s = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      float t = 0.0f;
#pragma unroll
      for (int b = 0; b < 4; ++b) t += w[b] * rf(2 * I - 1 + a, 2 * J - 1 + b);
      s += w[a] * t;
    }
    return 0.25f * s;
  }
  float s = 0.0f;
  for (int fi = 2 * I - 1; fi <= 2 * I + 2; ++fi) {
    if (fi < 0 || fi >= 2 * nxc) continue;
    const float wx = w1d(fi, I, nxc);
    float t = 0.0f;
    for (int fj = 2 * J - 1; fj <= 2 * J + 2; ++fj) {
      if (fj < 0 || fj >= 2 * nyc) continue;
      t += w1d(fj, J, nyc) * rf(fi, fj);
    }
    s += wx * t;
  }
  return 0.25f * s;
}

// prolongation P e at fine cell (fi, fj) of a coarse field read by ec(I, J)
template <typename F>
__device__ __forceinline__ float prolong_at(F ec, int fi, int fj, int nxc, int nyc) {
  const int ci = fi >> 1, cj = fj >> 1;
  const int sx = (fi & 1) ? 1 : -1, sy = (fj & 1) ? 1 : -1;
  float v = 0.0f;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    int ii = ci + ((s & 1) ? sx : 0), jj = cj + ((s & 2) ? sy : 0);
    float ww = (s == 0) ? 9.0f / 16.0f : ((s == 3) ? 1.0f / 16.0f : 3.0f / 16.0f);
    if (ii < 0 || ii >= nxc) { ii = ci; ww = -ww; }
    if (jj < 0 || jj >= nyc) { jj = cj; ww = -ww; }
    v += ww * ec(ii, jj);
  }
  return v;
}

__global__ void __launch_bounds__(NT)
restrict_kernel(const float* __restrict__ rf, float* __restrict__ fc, int nxc, int nyc) {
  const int nyf = 2 * nyc;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nxc * nyc;
       k += (long long)gridDim.x * NT) {
    const int I = (int)(k / nyc), J = (int)(k - (long long)I * nyc);
    fc[k] = restrict_at([&](int fi, int fj) { return rf[fi * nyf + fj]; }, I, J, nxc, nyc);
  }
}

__global__ void __launch_bounds__(NT)
prolong_add_kernel(const float* __restrict__ ec, float* __restrict__ xf, int nxc, int nyc) {
  const int nxf = 2 * nxc, nyf = 2 * nyc;
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nxf * nyf;
       k += (long long)gridDim.x * NT) {
    const int fi = (int)(k / nyf), fj = (int)(k - (long long)fi * nyf);
    xf[k] += prolong_at([&](int I, int J) { return ec[I * nyc + J]; }, fi, fj, nxc, nyc);
  }
}

// ── fused fine-level kernels: one launch per level on the way down and one on
// the way up.  A CTA owns a 32 x 32 tile and stages the tile plus a halo in
// shared memory; each red-black half-sweep is valid one cell further inside
// the staged region than the last, so after 2 nu half-sweeps the tile (plus
// the ring the residual and restriction need) holds exactly the values the
// level-wide sweeps produce.  The operator and update are the same float
// expressions as apply_at / rbgs_kernel, so the result is bit-identical to the
// one-kernel-per-sweep sequence.
constexpr int FT = 32;            // tile side of the levels with a tile for every SM
constexpr int FTS = 16;           // tile side of the smaller levels
// threads of a fused level CTA (one-dimensional): 256 for the 32^2 tiles, 512
// for the 16^2 ones; a compile-time count lets every phase's item loop have a
// fixed trip count
__host__ __device__ constexpr int fused_threads(int tile) { return tile == FT ? 256 : 512; }
// register cap of the level kernels: 64 per thread (four 256-thread CTAs per
// SM; capped for five CTAs, at 46-48 registers, the V-cycle ran 2 % slower)
constexpr int FNT_MAX = 1024;

// Staged layout of a tile with its ring: R = tile + 2 halo rows; the arrays
// x, f (the residual overwrites it), idg (R rows) and cx (R + 1 rows) keep PAD
// leading columns so that
// every staged row starts on a 16-byte boundary of the level's row (its first
// column j0 - halo - PAD is a multiple of 4) and a row stride RS, a multiple
// of 4 floats; cy (R rows of R + 1) stays unpadded.
__host__ __device__ constexpr int stage_pad(int halo) { return (4 - halo % 4) % 4; }
__host__ __device__ constexpr int stage_rs(int halo, int tile) {
  return ((tile + 2 * halo + stage_pad(halo) + 3) / 4) * 4;
}
// the up kernel's staged coarse tile (R / 2 + 2 square)
__host__ __device__ inline size_t up_tile_smem(int halo, int tile) {
  const int cr = (tile + 2 * halo) / 2 + 2;
  return (size_t)cr * cr * sizeof(float);
}
__host__ __device__ inline size_t fused_smem(int halo, int tile) {
  const int R = tile + 2 * halo, RS = stage_rs(halo, tile);
  return (size_t)(3 * R * RS + (R + 1) * RS + R * (R + 1)) * sizeof(float);
}

// 4-byte asynchronous global -> shared copy; src_bytes 0 writes a zero
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 4 : 0)
               : "memory");
}
// 16-byte version (four floats of a row; both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16f(float* dst, const float* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Shared-memory image of a level's tile plus a HALO-wide ring: x, f (r), idg
// (R x R) and the face coefficients cx ((R+1) x R), cy (R x (R+1)).  A tile
// whose ring lies wholly inside the level (most of them) takes the EDGE-free
// path: no domain tests and no Dirichlet ghosts.
template <int HALO, int TT>
struct Stage {
  static constexpr int R = TT + 2 * HALO;
  static constexpr int PAD = stage_pad(HALO);
  static constexpr int RS = stage_rs(HALO, TT);
  static constexpr int NTH = fused_threads(TT);
  // staged element (a, b) of x, f, idg (a in [0, R)) or cx (a in [0, R])
  __device__ static constexpr int at(int a, int b) { return a * RS + b + PAD; }
  int i0, j0, nx, ny;
  bool interior;
  float *x, *f, *r, *idg, *cx, *cy, *ec;
  __device__ bool inside(int a, int b) const {
    const int gi = i0 - HALO + a, gj = j0 - HALO + b;
    return gi >= 0 && gi < nx && gj >= 0 && gj < ny;
  }
  template <bool EDGE>
  __device__ float ax(int a, int b, float idx2) const {
    const float xc = x[at(a, b)];
    const float ea = cx[at(a + 1, b)], wa = cx[at(a, b)];
    const float nb = cy[a * (R + 1) + b + 1], sb = cy[a * (R + 1) + b];
    float xe = x[at(a + 1, b)], xw = x[at(a - 1, b)];
    float xn = x[at(a, b + 1)], xs = x[at(a, b - 1)];
    if (EDGE) {
      const int gi = i0 - HALO + a, gj = j0 - HALO + b;
      if (gi + 1 >= nx) xe = -xc;
      if (gi <= 0) xw = -xc;
      if (gj + 1 >= ny) xn = -xc;
      if (gj <= 0) xs = -xc;
    }
    return (ea * (xc - xe) + wa * (xc - xw) + nb * (xc - xn) + sb * (xc - xs)) * idx2;
  }
  // sum of c_f x_j over the in-domain neighbours (a wall's ghost belongs to
  // the diagonal)
  template <bool EDGE>
  __device__ float nbsum(int a, int b) const {
    const float ea = cx[at(a + 1, b)], wa = cx[at(a, b)];
    const float nb = cy[a * (R + 1) + b + 1], sb = cy[a * (R + 1) + b];
    float xe = x[at(a + 1, b)], xw = x[at(a - 1, b)];
    float xn = x[at(a, b + 1)], xs = x[at(a, b - 1)];
    if (EDGE) {
      const int gi = i0 - HALO + a, gj = j0 - HALO + b;
      if (gi + 1 >= nx) xe = 0.0f;
      if (gi <= 0) xw = 0.0f;
      if (gj + 1 >= ny) xn = 0.0f;
      if (gj <= 0) xs = 0.0f;
    }
    return (ea * xe + wa * xw) + (nb * xn + sb * xs);
  }
  // red-black update x_i = (f_i + idx2 sum_j c_ij x_j) / d_i (the same update
  // as x_i += (f_i - (A x)_i) / d_i, with d_i's inverse staged)
  template <bool EDGE>
  __device__ void sweep_impl(int color, int m, float idx2) const {
    for (int a = m + (int)threadIdx.y; a < R - m; a += (int)blockDim.y) {
      const int gi = i0 - HALO + a;
      // first column b >= m with (gi + gj) % 2 == color, gj = j0 - HALO + b
      int b = m + (((color - gi - (j0 - HALO) - m) % 2 + 2) % 2) + 2 * (int)threadIdx.x;
      for (; b < R - m; b += 2 * (int)blockDim.x) {
        if (EDGE && !inside(a, b)) continue;
        x[at(a, b)] = (f[at(a, b)] + nbsum<EDGE>(a, b) * idx2) * idg[at(a, b)];
      }
    }
    __syncthreads();
  }
  // the first half-sweep of a V-cycle's way down starts from x = 0, where
  // A x = 0 exactly: the update is x = f / d
  // (the cells enumerated as in sweep_flat, margin 1)
  __device__ void sweep_from_zero(int color) const {
    constexpr int M = 1, NR = R - 2 * M, HALF = NR / 2;
#pragma unroll
    for (int e = (int)threadIdx.x; e < NR * HALF; e += NTH) {
      const int a = M + e / HALF, k = e - (e / HALF) * HALF;
      // tile origins are even, so the colour of staged (a, b) is (a + b) % 2
      const int b = M + ((color + a + M) & 1) + 2 * k;
      if (!interior && !inside(a, b)) continue;
      x[at(a, b)] = f[at(a, b)] * idg[at(a, b)];
    }
    __syncthreads();
  }
  // The same half-sweep with the cells of `color` at least M cells inside
  // the staged region enumerated as one list over all the threads (NR / 2 of
  // them in each of the NR rows), so that no lane idles at the ends of the
  // rows (a row of 44 cells has 22 of a colour for 32 lanes)
  template <bool EDGE, int M>
  __device__ void sweep_flat(int color, float idx2) const {
    constexpr int NR = R - 2 * M, HALF = NR / 2;
#pragma unroll
    for (int e = (int)threadIdx.x; e < NR * HALF; e += NTH) {
      const int a = M + e / HALF, k = e - (e / HALF) * HALF;
      // tile origins are even, so the colour of staged (a, b) is (a + b) % 2
      const int b = M + ((color + a + M) & 1) + 2 * k;
      if (EDGE && !inside(a, b)) continue;
      x[at(a, b)] = (f[at(a, b)] + nbsum<EDGE>(a, b) * idx2) * idg[at(a, b)];
    }
    __syncthreads();
  }
  template <bool EDGE>
  __device__ void sweep_m(int color, int m, float idx2) const {
    switch (m) {
#define ZB_SWEEP_M(M) \
  case M: if constexpr (R - 2 * M >= 2) { sweep_flat<EDGE, M>(color, idx2); return; } break;
      ZB_SWEEP_M(1) ZB_SWEEP_M(2) ZB_SWEEP_M(3) ZB_SWEEP_M(4) ZB_SWEEP_M(5)
      ZB_SWEEP_M(6) ZB_SWEEP_M(7) ZB_SWEEP_M(8) ZB_SWEEP_M(9)
#undef ZB_SWEEP_M
      default: break;
    }
    sweep_impl<EDGE>(color, m, idx2);
  }
  // one half-sweep over the cells of `color` at least m cells inside the
  // staged region
  __device__ void sweep(int color, int m, float idx2) const {
    if (interior) sweep_m<false>(color, m, idx2);
    else sweep_m<true>(color, m, idx2);
  }
  __device__ float residual(int a, int b, float idx2) const {
    if (interior) return f[at(a, b)] - ax<false>(a, b, idx2);
    return inside(a, b) ? f[at(a, b)] - ax<true>(a, b, idx2) : 0.0f;
  }
};

template <int HALO, int TT>
__device__ Stage<HALO, TT> stage_level(float* sm, int i0, int j0, int nx, int ny,
                                       const float* __restrict__ f, const float* __restrict__ cx,
                                       const float* __restrict__ cy, const float* __restrict__ idg,
                                       const float* __restrict__ x, int vec,
                                       const float* __restrict__ ec = nullptr) {
  using St = Stage<HALO, TT>;
  constexpr int R = St::R, RS = St::RS, PAD = St::PAD;
  St S;
  S.i0 = i0; S.j0 = j0; S.nx = nx; S.ny = ny;
  S.interior = i0 - HALO >= 0 && j0 - HALO >= 0 && i0 - HALO + R <= nx && j0 - HALO + R <= ny;
  // the residual overwrites f in place (a cell's residual reads only its own
  // f), so r shares f's array
  S.x = sm; S.f = sm + R * RS; S.r = S.f; S.idg = sm + 2 * R * RS;
  S.cx = sm + 3 * R * RS; S.cy = S.cx + (R + 1) * RS;
  S.ec = S.cy + R * (R + 1);
  constexpr int nt = St::NTH;
  const int tid = threadIdx.x;
  // every copy is issued before any is waited for
  if (vec) {
    // rows as 16-byte chunks from column gs = j0 - HALO - PAD (a multiple of
    // 4, like ny): a chunk lies wholly inside the level or wholly outside it.
    // Each thread keeps one chunk column and steps down the rows.
    constexpr int NC = RS / 4, RSTEP = nt / NC;
    const int c = tid % NC, a0 = tid / NC;
    if (a0 < RSTEP) {
      const int gc = j0 - HALO - PAD + 4 * c;
      const bool cin = gc >= 0 && gc < ny;
      const int gi0 = i0 - HALO + a0;
      const long long k0 = (long long)gi0 * ny + gc;
#pragma unroll
      for (int it = 0; it < (R + RSTEP - 1) / RSTEP; ++it) {
        const int a = a0 + it * RSTEP, gi = gi0 + it * RSTEP;
        if (a < R) {
          const bool in = cin && gi >= 0 && gi < nx;
          const long long k = in ? k0 + (long long)it * RSTEP * ny : 0;
          cp_async16f(S.f + a * RS + 4 * c, f + k, in);
          cp_async16f(S.idg + a * RS + 4 * c, idg + k, in);
          if (x) cp_async16f(S.x + a * RS + 4 * c, x + k, in);
          else *(float4*)(S.x + a * RS + 4 * c) = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
#pragma unroll
      for (int it = 0; it < (R + 1 + RSTEP - 1) / RSTEP; ++it) {
        const int a = a0 + it * RSTEP, gi = gi0 + it * RSTEP;
        if (a < R + 1) {
          const bool in = cin && gi >= 0 && gi <= nx;
          const long long k = in ? k0 + (long long)it * RSTEP * ny : 0;
          cp_async16f(S.cx + a * RS + 4 * c, cx + k, in);
        }
      }
    }
  } else {
#pragma unroll
    for (int e = tid; e < R * R; e += nt) {
      const int a = e / R, b = e - (e / R) * R;
      const int gi = i0 - HALO + a, gj = j0 - HALO + b;
      const bool in = gi >= 0 && gi < nx && gj >= 0 && gj < ny;
      const long long k = in ? (long long)gi * ny + gj : 0;
      cp_async4(S.f + St::at(a, b), f + k, in);
      cp_async4(S.idg + St::at(a, b), idg + k, in);
      if (x) cp_async4(S.x + St::at(a, b), x + k, in);
      else S.x[St::at(a, b)] = 0.0f;
    }
#pragma unroll
    for (int e = tid; e < (R + 1) * R; e += nt) {
      const int a = e / R, b = e - (e / R) * R;
      const int gi = i0 - HALO + a, gj = j0 - HALO + b;
      const bool in = gi >= 0 && gi <= nx && gj >= 0 && gj < ny;
      cp_async4(S.cx + St::at(a, b), cx + (in ? (long long)gi * ny + gj : 0), in);
    }
  }
  // cy: R rows of R + 1 faces, 4-byte copies (rows of ny + 1 floats do not
  // start on 16 bytes); each thread keeps one column and steps down the rows
  {
    constexpr int W = R + 1, YSTEP = nt / W;
    const int b = tid % W, a0 = tid / W;
    if (a0 < YSTEP) {
      const int gj = j0 - HALO + b, gi0 = i0 - HALO + a0;
      const bool cin = gj >= 0 && gj <= ny;
      const long long k0 = (long long)gi0 * (ny + 1) + gj;
#pragma unroll
      for (int it = 0; it < (R + YSTEP - 1) / YSTEP; ++it) {
        const int a = a0 + it * YSTEP, gi = gi0 + it * YSTEP;
        if (a < R) {
          const bool in = cin && gi >= 0 && gi < nx;
          cp_async4(S.cy + a * W + b, cy + (in ? k0 + (long long)it * YSTEP * (ny + 1) : 0), in);
        }
      }
    }
  }
  if (ec) {
    // the coarse level's result under the tile (coarse cells I0 - 1 ..
    // I0 + R / 2, I0 = (i0 - HALO) / 2, and the same in y), loaded while the
    // copies fly; a coarse index one beyond the wall holds the prolongation's
    // odd reflection (minus the cell inside; plus it at a corner), so the
    // correction below needs no wall tests; cells further out are never read
    constexpr int CR = R / 2 + 2;
    const int nxc = nx / 2, nyc = ny / 2;
    const int I0 = (i0 - HALO) / 2 - 1, J0 = (j0 - HALO) / 2 - 1;
#pragma unroll
    for (int e = tid; e < CR * CR; e += nt) {
      const int ci = I0 + e / CR, cj = J0 + e % CR;
      float v = 0.0f;
      if (ci >= -1 && ci <= nxc && cj >= -1 && cj <= nyc) {
        const bool ox = ci < 0 || ci >= nxc, oy = cj < 0 || cj >= nyc;
        const int ri = ci < 0 ? 0 : (ci >= nxc ? nxc - 1 : ci);
        const int rj = cj < 0 ? 0 : (cj >= nyc ? nyc - 1 : cj);
        v = ec[(long long)ri * nyc + rj];
        if (ox != oy) v = -v;
      }
      S.ec[e] = v;
    }
  }
  cp_async_wait_all();
  __syncthreads();
  return S;
}

// pre-smoothing from x = 0 (NU red/black pairs), residual, restriction:
// writes the tile's x and the coarse right-hand side of its TT/2 x TT/2
// coarse cells
template <int NU, int TT>
__global__ void __launch_bounds__(FNT_MAX)
mg_down_kernel(const float* __restrict__ f, const float* __restrict__ cx,
               const float* __restrict__ cy, const float* __restrict__ idg, float* __restrict__ x,
               float* __restrict__ fc, int nx, int ny, float idx2, int vec) {
  pdl_enter();
  extern __shared__ float fsm[];
  constexpr int HALO = 2 * NU + 2;
  constexpr int R = Stage<HALO, TT>::R;
  const int i0 = blockIdx.y * TT, j0 = blockIdx.x * TT;
  constexpr int nt = fused_threads(TT);
  const int tid = threadIdx.x;
  const Stage<HALO, TT> S = stage_level<HALO, TT>(fsm, i0, j0, nx, ny, f, cx, cy, idg, nullptr, vec);
  if (NU > 0) S.sweep_from_zero(0);
  for (int s = 1; s < 2 * NU; ++s) S.sweep(s & 1, s + 1, idx2);
  // residual where the sweeps are final and one ring beyond the tile (one
  // list of cells over all the threads)
  {
    constexpr int m = 2 * NU + 1, NRr = R - 2 * m;
#pragma unroll
    for (int e = tid; e < NRr * NRr; e += nt) {
      const int a = m + e / NRr, b = m + (e - (e / NRr) * NRr);
      S.r[S.at(a, b)] = S.residual(a, b, idx2);
    }
  }
  __syncthreads();
#pragma unroll
  for (int e = tid; e < TT * TT; e += nt) {
    const int ti = e / TT, tj = e % TT;
    const int gi = i0 + ti, gj = j0 + tj;
    if (gi < nx && gj < ny) x[(long long)gi * ny + gj] = S.x[S.at(HALO + ti, HALO + tj)];
  }
  const int nxc = nx / 2, nyc = ny / 2;
#pragma unroll
  for (int e = tid; e < (TT / 2) * (TT / 2); e += nt) {
    const int I = i0 / 2 + e / (TT / 2), J = j0 / 2 + e % (TT / 2);
    if (I >= nxc || J >= nyc) continue;
    fc[(long long)I * nyc + J] = restrict_at(
        [&](int fi, int fj) { return S.r[S.at(fi - i0 + HALO, fj - j0 + HALO)]; }, I, J, nxc,
        nyc);
  }
}

// x += P e (coarse correction), post-smoothing (NU black/red pairs).  The
// tile stages its halo from `x` (the way down's result, which neighbouring
// tiles also read) and writes the level's result to the separate `xo`: a tile
// that finished before a neighbour staged its halo must not have overwritten
// what that neighbour reads (a level with more tiles than one wave of CTAs)
template <int NU, int TT>
__global__ void __launch_bounds__(FNT_MAX)
mg_up_kernel(const float* __restrict__ f, const float* __restrict__ cx,
             const float* __restrict__ cy, const float* __restrict__ idg,
             const float* __restrict__ x, const float* __restrict__ ec, float* __restrict__ xo,
             int nx, int ny, float idx2, int vec) {
  pdl_enter();
  extern __shared__ float fsm[];
  constexpr int HALO = 2 * NU;
  constexpr int R = Stage<HALO, TT>::R;
  const int i0 = blockIdx.y * TT, j0 = blockIdx.x * TT;
  constexpr int nt = fused_threads(TT);
  const int tid = threadIdx.x;
  const Stage<HALO, TT> S =
      stage_level<HALO, TT>(fsm, i0, j0, nx, ny, f, cx, cy, idg, x, vec, ec);
  // coarse correction: each coarse cell under the staged region adds its
  // prolongation to its 2 x 2 fine children -- prolong_at's weights in its
  // order (own 9/16, x side 3/16, y side 3/16, diagonal 1/16), the wall
  // reflection staged -- so the sums are prolong_at's bits.  Children outside
  // the level are updated too; nothing reads them.
  {
    constexpr int CR = R / 2 + 2, NP = R / 2;
    const float* T = S.ec;
#pragma unroll
    for (int e = tid; e < NP * NP; e += nt) {
      const int p = 1 + e / NP, q = 1 + e % NP;
      const float c0 = T[p * CR + q];
      const float xm = T[(p - 1) * CR + q], xp = T[(p + 1) * CR + q];
      const float ym = T[p * CR + q - 1], yp = T[p * CR + q + 1];
      const float mm = T[(p - 1) * CR + q - 1], mp = T[(p - 1) * CR + q + 1];
      const float pm = T[(p + 1) * CR + q - 1], pp = T[(p + 1) * CR + q + 1];
#pragma unroll
      for (int d = 0; d < 4; ++d) {
        const int di = d >> 1, dj = d & 1;
        const float ex = di ? xp : xm, ey = dj ? yp : ym;
        const float exy = di ? (dj ? pp : pm) : (dj ? mp : mm);
        float v = 0.0f;
        v += (9.0f / 16.0f) * c0;
        v += (3.0f / 16.0f) * ex;
        v += (3.0f / 16.0f) * ey;
        v += (1.0f / 16.0f) * exy;
        S.x[S.at(2 * p - 2 + di, 2 * q - 2 + dj)] += v;
      }
    }
  }
  __syncthreads();
  for (int s = 0; s < 2 * NU; ++s) S.sweep(1 - (s & 1), s + 1, idx2);
#pragma unroll
  for (int e = tid; e < TT * TT; e += nt) {
    const int ti = e / TT, tj = e % TT;
    const int gi = i0 + ti, gj = j0 + tj;
    if (gi < nx && gj < ny) xo[(long long)gi * ny + gj] = S.x[S.at(HALO + ti, HALO + tj)];
  }
}

__global__ void zero32_kernel(float* x, long long n) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT)
    x[k] = 0.0f;
}

__global__ void copy32_kernel(const float* a, float* b, long long n) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT)
    b[k] = a[k];
}

// ── the one-CTA coarse V-cycle (levels small0 .. nlev-1 in shared memory) ───
// Every level of at most 32 x 32 cells runs with one thread per cell: thread t
// holds cell (t >> sh, t & (2^sh - 1)), 2^sh the level's row length rounded up
// to a power of two, so no thread divides, and a red-black half-sweep gives
// each thread one cell of the colour (rows of 2^(sh-1) threads).  A level's
// phases synchronise only the warps that hold its cells (a named barrier per
// level; a warp barrier for a one-warp level): the coarser levels run in a few
// warps while the others wait at the next finer level's barrier.  Everything
// the cycle reads (coefficients, inverse diagonals, the coarsest inverse, the
// right-hand side) is staged by one round of asynchronous copies.  The sums are
// the same float expressions as the level-wide kernels', so the result is the
// same bits.
constexpr int CT = 1024;
constexpr int CT_MAX_LEVELS = 15;   // named barriers 1 .. 15, one per level

struct CLevel {
  int nx, ny, sh, act;        // act: threads holding the level's cells (multiple of 32)
  float idx2;
  int x, f, r, cx, cy, idg;   // float offsets into shared memory
};

__device__ __forceinline__ void level_sync(int id, int act) {
  if (act <= 32) __syncwarp();
  else asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(act) : "memory");
}

// one half-sweep of `color` by thread t; from_zero: the level's x is zero
// before it (the neighbour sum is then 0, and x need not be cleared)
__device__ __forceinline__ void cl_half(float* sm, const CLevel& c, int t, int color,
                                        bool from_zero) {
  const int hs = c.sh > 0 ? c.sh - 1 : 0;
  const int i = t >> hs, m = t & ((1 << hs) - 1);
  const int j = 2 * m + ((i + color) & 1);
  if (i < c.nx && j < c.ny) {
    const int k = i * c.ny + j;
    const float nb = from_zero ? 0.0f : nbsum_at(sm + c.x, sm + c.cx, sm + c.cy, c.nx, c.ny, i, j);
    sm[c.x + k] = (sm[c.f + k] + c.idx2 * nb) * sm[c.idg + k];
  }
}

__global__ void __launch_bounds__(CT)
coarse_vcycle_kernel(const Plan P, float* ws_f, int nu, int coarse_sweeps) {
  pdl_enter();
  extern __shared__ float sm[];
  __shared__ CLevel tab[MAXL];
  const int t = threadIdx.x;
  const int l0 = P.small0, nl = P.nlev;
  // shared layout, level after level: x, f, r (n each), cx, cy, idg; then the
  // coarsest inverse with rows padded to n + 1 (no bank conflicts)
  int inv_off = 0;
  for (int l = l0; l < nl; ++l) {
    const Level& L = P.L[l];
    const int n = L.nx * L.ny;
    if (t == l - l0) {
      CLevel c;
      c.nx = L.nx;
      c.ny = L.ny;
      int sh = 0;
      while ((1 << sh) < L.ny) ++sh;
      c.sh = sh;
      c.act = ((L.nx << sh) + 31) & ~31;
      c.idx2 = 1.0f / (L.dx * L.dx);
      c.x = inv_off;
      c.f = c.x + n;
      c.r = c.f + n;
      c.cx = c.r + n;
      c.cy = c.cx + (L.nx + 1) * L.ny;
      c.idg = c.cy + L.nx * (L.ny + 1);
      tab[l] = c;
    }
    inv_off += 4 * n + (L.nx + 1) * L.ny + L.nx * (L.ny + 1);
  }
  const Level& Lc = P.L[nl - 1];
  const int nc = Lc.nx * Lc.ny;
  float* sinv = sm + inv_off;
  __syncthreads();
  for (int l = l0; l < nl; ++l) {
    const Level& L = P.L[l];
    const CLevel c = tab[l];
    const int n = L.nx * L.ny;
    for (int k = t; k < (L.nx + 1) * L.ny; k += CT) cp_async4(sm + c.cx + k, ws_f + L.cx + k, true);
    for (int k = t; k < L.nx * (L.ny + 1); k += CT) cp_async4(sm + c.cy + k, ws_f + L.cy + k, true);
    for (int k = t; k < n; k += CT) cp_async4(sm + c.idg + k, ws_f + L.idg + k, true);
    if (l == l0)
      for (int k = t; k < n; k += CT) cp_async4(sm + c.f + k, ws_f + L.f + k, true);
  }
  if (P.cinv >= 0)
    for (int k = t; k < nc * nc; k += CT) {
      const int a = k / nc, b = k - a * nc;
      cp_async4(sinv + a * (nc + 1) + b, ws_f + P.cinv + k, true);
    }
  cp_async_wait_all();
  __syncthreads();
  // The first level's cell of each thread keeps its operands in registers for
  // the whole cycle (its faces, inverse diagonal and right-hand side do not
  // change): its half-sweeps and residual then read only the neighbours' x,
  // with nbsum_at's and apply_at's expressions in their order
  const CLevel c0 = tab[l0];
  const int i0c = t >> c0.sh, j0c = t & ((1 << c0.sh) - 1);
  const bool own0 = t < c0.act && i0c < c0.nx && j0c < c0.ny;
  const int k0c = own0 ? i0c * c0.ny + j0c : 0;
  float ce = 0.0f, cw = 0.0f, cn = 0.0f, cs = 0.0f, f0c = 0.0f, g0c = 0.0f;
  if (own0) {
    ce = sm[c0.cx + (i0c + 1) * c0.ny + j0c];
    cw = sm[c0.cx + i0c * c0.ny + j0c];
    cn = sm[c0.cy + i0c * (c0.ny + 1) + j0c + 1];
    cs = sm[c0.cy + i0c * (c0.ny + 1) + j0c];
    f0c = sm[c0.f + k0c];
    g0c = sm[c0.idg + k0c];
  }
  const bool hasE = i0c + 1 < c0.nx, hasW = i0c > 0, hasN = j0c + 1 < c0.ny, hasS = j0c > 0;
  float* const x0 = sm + c0.x;
  // half-sweep of `color` on the first level
  auto half0 = [&](int color, bool from_zero) {
    if (own0 && ((i0c + j0c + color) & 1) == 0) {
      float nb = 0.0f;
      if (!from_zero) {
        const float xe = hasE ? x0[k0c + c0.ny] : 0.0f, xw = hasW ? x0[k0c - c0.ny] : 0.0f;
        const float xn = hasN ? x0[k0c + 1] : 0.0f, xs = hasS ? x0[k0c - 1] : 0.0f;
        nb = (ce * xe + cw * xw) + (cn * xn + cs * xs);
      }
      x0[k0c] = (f0c + c0.idx2 * nb) * g0c;
    }
  };
  // descend: pre-smoothing, residual, restriction into the next level's f
  for (int l = l0; l < nl - 1; ++l) {
    const CLevel c = tab[l];
    const int id = 1 + l - l0;
    if (t < c.act) {
      if (l == l0) {
        for (int s = 0; s < nu; ++s) {
          half0(0, s == 0);
          level_sync(id, c.act);
          half0(1, false);
          level_sync(id, c.act);
        }
        if (own0) {
          const float xc = x0[k0c];
          const float xe = hasE ? x0[k0c + c0.ny] : -xc, xw = hasW ? x0[k0c - c0.ny] : -xc;
          const float xn = hasN ? x0[k0c + 1] : -xc, xs = hasS ? x0[k0c - 1] : -xc;
          sm[c0.r + k0c] =
              f0c - (ce * (xc - xe) + cw * (xc - xw) + cn * (xc - xn) + cs * (xc - xs)) * c0.idx2;
        }
      } else {
        for (int s = 0; s < nu; ++s) {
          cl_half(sm, c, t, 0, s == 0);
          level_sync(id, c.act);
          cl_half(sm, c, t, 1, false);
          level_sync(id, c.act);
        }
        const int i = t >> c.sh, j = t & ((1 << c.sh) - 1);
        if (i < c.nx && j < c.ny) {
          float od;
          sm[c.r + i * c.ny + j] =
              sm[c.f + i * c.ny + j] - apply_at(sm + c.x, sm + c.cx, sm + c.cy, c.nx, c.ny, i, j,
                                                c.idx2, od);
        }
      }
      level_sync(id, c.act);
      const CLevel cc = tab[l + 1];
      {
        const int I = t >> cc.sh, J = t & ((1 << cc.sh) - 1);
        if (I < cc.nx && J < cc.ny) {
          const float* rl = sm + c.r;
          const int nyf = c.ny;
          sm[cc.f + I * cc.ny + J] = restrict_at(
              [&](int fi, int fj) { return rl[fi * nyf + fj]; }, I, J, cc.nx, cc.ny);
        }
      }
      level_sync(id, c.act);
    }
  }
  // coarsest level: the dense inverse, else symmetric red-black sweep pairs
  {
    const CLevel c = tab[nl - 1];
    const int id = nl - l0;
    if (t < c.act) {
      if (P.cinv >= 0) {
        if (t < nc) {
          float v = 0.0f;
          for (int m = 0; m < nc; ++m) v += sinv[t * (nc + 1) + m] * sm[c.f + m];
          sm[c.x + t] = v;
        }
        level_sync(id, c.act);
      } else {
        for (int s = 0; s < coarse_sweeps; ++s) {
          cl_half(sm, c, t, 0, s == 0);
          level_sync(id, c.act);
          cl_half(sm, c, t, 1, false);
          level_sync(id, c.act);
        }
        for (int s = 0; s < coarse_sweeps; ++s) {
          cl_half(sm, c, t, 1, false);
          level_sync(id, c.act);
          cl_half(sm, c, t, 0, false);
          level_sync(id, c.act);
        }
      }
    }
  }
  // ascend: wait for the coarser level's result (its warps arrive after their
  // own phases), coarse correction, post-smoothing
  for (int l = nl - 2; l >= l0; --l) {
    const CLevel c = tab[l], cc = tab[l + 1];
    const int id = 1 + l - l0;
    if (t < c.act) {
      level_sync(id, c.act);
      {
        const int i = t >> c.sh, j = t & ((1 << c.sh) - 1);
        if (i < c.nx && j < c.ny) {
          const float* ecl = sm + cc.x;
          const int nyc = cc.ny;
          sm[c.x + i * c.ny + j] +=
              prolong_at([&](int I, int J) { return ecl[I * nyc + J]; }, i, j, cc.nx, cc.ny);
        }
      }
      level_sync(id, c.act);
      for (int s = 0; s < nu; ++s) {
        if (l == l0) half0(1, false);
        else cl_half(sm, c, t, 1, false);
        level_sync(id, c.act);
        if (l == l0) half0(0, false);
        else cl_half(sm, c, t, 0, false);
        level_sync(id, c.act);
      }
    }
  }
  __syncthreads();
  const Level& L0 = P.L[l0];
  for (int k = t; k < L0.nx * L0.ny; k += CT) ws_f[L0.xo + k] = sm[c0.x + k];
}

// The small levels' set-up in one CTA: levels l_first .. nlev - 1 coarsened
// one after the other (coarsen_cell per coarse cell), then the dense inverse of
// the coarsest operator (float64 in-place Gauss-Jordan; the operator is SPD, so
// no pivoting), stored as float32 for the V-cycle
constexpr int ST = 1024;
__global__ void __launch_bounds__(ST) small_setup_kernel(const Plan P, float* ws_f, int l_first) {
  __shared__ double a[DENSE_MAX_CELLS][DENSE_MAX_CELLS];
  __shared__ double fcol[DENSE_MAX_CELLS];
  __shared__ double prow[DENSE_MAX_CELLS];
  for (int l = l_first; l < P.nlev; ++l) {
    const Level& L = P.L[l];
    const Level& Lf = P.L[l - 1];
    // the host's IEEE quotient, as the launches of the larger levels get it
    const float idx2 = __fdiv_rn(1.0f, __fmul_rn(L.dx, L.dx));
    for (int k = threadIdx.x; k < L.nx * L.ny; k += ST) {
      const int I = k / L.ny, J = k - (k / L.ny) * L.ny;
      coarsen_cell(ws_f + Lf.cx, ws_f + Lf.cy, L.nx, L.ny, idx2, ws_f + L.cx, ws_f + L.cy,
                   ws_f + L.idg, I, J);
    }
    __syncthreads();
  }
  if (P.cinv < 0) return;
  const Level& L = P.L[P.nlev - 1];
  const int nx = L.nx, ny = L.ny, n = nx * ny;
  const double idx2 = 1.0 / ((double)L.dx * (double)L.dx);
  const float* cx = ws_f + L.cx;
  const float* cy = ws_f + L.cy;
  for (int e = threadIdx.x; e < n * n; e += ST) a[e / n][e % n] = 0.0;
  __syncthreads();
  // row k of the operator, one thread per row
  for (int k = threadIdx.x; k < n; k += ST) {
    const int i = k / ny, j = k - (k / ny) * ny;
    const double e = cx[(i + 1) * ny + j], w = cx[i * ny + j];
    const double nn = cy[i * (ny + 1) + j + 1], ss = cy[i * (ny + 1) + j];
    double d = (e + w) + (nn + ss);
    if (i == 0) d += w;
    if (i == nx - 1) d += e;
    if (j == 0) d += ss;
    if (j == ny - 1) d += nn;
    a[k][k] = d * idx2;
    if (i + 1 < nx) a[k][k + ny] = -e * idx2;
    if (i > 0) a[k][k - ny] = -w * idx2;
    if (j + 1 < ny) a[k][k + 1] = -nn * idx2;
    if (j > 0) a[k][k - 1] = -ss * idx2;
  }
  __syncthreads();
  // two phases per pivot, each only reading what the previous phase wrote:
  // (1) the scaled pivot row and the pivot column go to side arrays, (2) the
  // rank-one update writes every row
  for (int p = 0; p < n; ++p) {
    for (int c = threadIdx.x; c < n; c += ST) prow[c] = (c == p ? 1.0 : a[p][c]) / a[p][p];
    for (int r = threadIdx.x; r < n; r += ST) fcol[r] = (r == p) ? 0.0 : a[r][p];
    __syncthreads();
    for (int e = threadIdx.x; e < n * n; e += ST) {
      const int r = e / n, c = e % n;
      a[r][c] = (r == p) ? prow[c] : (c == p ? 0.0 : a[r][c]) - fcol[r] * prow[c];
    }
    __syncthreads();
  }
  float* inv = ws_f + P.cinv;
  for (int e = threadIdx.x; e < n * n; e += ST) inv[e] = (float)a[e / n][e % n];
}

// the one-CTA kernel's dynamic shared memory at most: 227 KB less its static
// level table
constexpr size_t COARSE_SMEM_MAX = 227 * 1024 - sizeof(CLevel) * MAXL;

static size_t coarse_smem(const Plan& P) {
  size_t o = 0;
  for (int l = P.small0; l < P.nlev; ++l) {
    const Level& L = P.L[l];
    const size_t n = (size_t)L.nx * L.ny;
    o += 4 * n + (size_t)(L.nx + 1) * L.ny + (size_t)L.nx * (L.ny + 1);
  }
  if (P.cinv >= 0) {
    const size_t nc = (size_t)P.L[P.nlev - 1].nx * P.L[P.nlev - 1].ny;
    o += nc * (nc + 1);
  }
  return o * sizeof(float);
}

// opt the one-CTA kernel into the full 227 KB of shared memory (once per
// device; called from set-up, never inside a stream capture)
static int enable_coarse_smem() {
  static std::atomic<unsigned> set_mask{0u};
  int dev = 0;
  ZB_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 32 && !(set_mask.load() & (1u << dev))) {
    ZB_CUDA_TRY(cudaFuncSetAttribute(coarse_vcycle_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)COARSE_SMEM_MAX));
#define ZB_SMEM_ATTR(K) \
    ZB_CUDA_TRY(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024))
    ZB_SMEM_ATTR((mg_down_kernel<1, FT>)); ZB_SMEM_ATTR((mg_down_kernel<2, FT>));
    ZB_SMEM_ATTR((mg_down_kernel<3, FT>)); ZB_SMEM_ATTR((mg_down_kernel<4, FT>));
    ZB_SMEM_ATTR((mg_up_kernel<1, FT>)); ZB_SMEM_ATTR((mg_up_kernel<2, FT>));
    ZB_SMEM_ATTR((mg_up_kernel<3, FT>)); ZB_SMEM_ATTR((mg_up_kernel<4, FT>));
    ZB_SMEM_ATTR((mg_down_kernel<1, FTS>)); ZB_SMEM_ATTR((mg_down_kernel<2, FTS>));
    ZB_SMEM_ATTR((mg_down_kernel<3, FTS>)); ZB_SMEM_ATTR((mg_down_kernel<4, FTS>));
    ZB_SMEM_ATTR((mg_up_kernel<1, FTS>)); ZB_SMEM_ATTR((mg_up_kernel<2, FTS>));
    ZB_SMEM_ATTR((mg_up_kernel<3, FTS>)); ZB_SMEM_ATTR((mg_up_kernel<4, FTS>));
#undef ZB_SMEM_ATTR
    set_mask.fetch_or(1u << dev);
  }
  return ZB_OK;
}

// the graph solve's loop control, folded into the last kernel of the start
// and of every iteration (nullptr: none, the host drives the loop)
struct LoopCtl {
  cudaGraphConditionalHandle h;
  double tol;
  int maxit;
};

// reduction counters of finish_scalars: four unsigned slots in the last
// doubles of the scalar block (zeroed at set-up, re-armed by every use)
static unsigned* counters(double* scal) { return (unsigned*)(scal + 12); }

static int grid_for(long long n) {
  return (int)std::max<long long>(1, std::min<long long>((n + NT - 1) / NT, 148 * 8));
}

}  // namespace pois
}  // namespace zb

// ── coupling to the SWE state: right-hand side and corrector ────────────────
namespace zb {
namespace pois {

template <typename T>
__global__ void rhs_kernel(const T* __restrict__ qx, const T* __restrict__ qy, int nx, int ny,
                           double inv_dt_dx, double* __restrict__ b) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    const double qc = (double)qx[k], pc = (double)qy[k];
    const double fe = i + 1 < nx ? 0.5 * (qc + (double)qx[k + ny]) : 0.0;
    const double fw = i > 0 ? 0.5 * ((double)qx[k - ny] + qc) : 0.0;
    const double fn = j + 1 < ny ? 0.5 * (pc + (double)qy[k + 1]) : 0.0;
    const double fs = j > 0 ? 0.5 * ((double)qy[k - 1] + pc) : 0.0;
    b[k] = -((fe - fw) + (fn - fs)) * inv_dt_dx;
  }
}

template <typename T>
__global__ void correct_kernel(T* __restrict__ qx, T* __restrict__ qy,
                               const double* __restrict__ cx, const double* __restrict__ cy,
                               const double* __restrict__ p, int nx, int ny, double dt,
                               double inv_dx) {
  for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < (long long)nx * ny;
       k += (long long)gridDim.x * NT) {
    const int i = (int)(k / ny), j = (int)(k - (long long)i * ny);
    const double pc = p[k];
    const double gw = cx[(long long)i * ny + j] * (pc - ghost_or(p, nx, ny, i - 1, j, pc)) * inv_dx;
    const double ge = cx[(long long)(i + 1) * ny + j] * (ghost_or(p, nx, ny, i + 1, j, pc) - pc) * inv_dx;
    const double gs = cy[(long long)i * (ny + 1) + j] * (pc - ghost_or(p, nx, ny, i, j - 1, pc)) * inv_dx;
    const double gn = cy[(long long)i * (ny + 1) + j + 1] * (ghost_or(p, nx, ny, i, j + 1, pc) - pc) * inv_dx;
    qx[k] = (T)((double)qx[k] - dt * 0.5 * (gw + ge));
    qy[k] = (T)((double)qy[k] - dt * 0.5 * (gs + gn));
  }
}

static bool valid(const zb_poisson_cfg* c) {
  return c && c->nx >= 2 && c->ny >= 2 && c->dx > 0 && c->cmin > 0 && c->cmax >= c->cmin &&
         c->nu >= 0 && c->nu <= 4 && c->coarse_sweeps >= 1 && c->coarsest >= 2 &&
         (long long)c->nx * c->ny < (1LL << 31);
}

// z32 = M r32 on level 0 (f0 already holds r); precond: 0 none, 1 MG, 2 MG
// followed by one learned smoothing step on level 0 (x += S(f - A x)), 3 MG
// with the level-0 red-black smoothing replaced by the learned smoother
// One fused level launch (down: pre-smoothing, residual, restriction into the
// coarse right-hand side `to`; up: coarse correction from `to`, post-smoothing)
// with TT x TT tiles.
template <int TT>
static int fused_level(bool down, int nu, const Level& L, float* fw, float* to, float idx2,
                       dim3 blk, cudaStream_t st) {
  // down: `to` = the coarse right-hand side it restricts into; up: `to` =
  // the coarse level's result it prolongs from
  const dim3 grid((L.ny + TT - 1) / TT, (L.nx + TT - 1) / TT);
  const size_t sm = down ? fused_smem(2 * nu + 2, TT) : fused_smem(2 * nu, TT) + up_tile_smem(2 * nu, TT);
  const float *a0 = fw + L.f, *a1 = fw + L.cx, *a2 = fw + L.cy, *a3 = fw + L.idg;
  float* a4 = fw + L.x;
  float* a5 = fw + L.xo;
  // rows staged as 16-byte chunks when every staged array is 16-byte aligned
  // and the level's rows are a multiple of 4 floats (the plan aligns the
  // arrays; odd-sized coarse levels take the 4-byte copies)
  auto al16 = [](const void* p) { return ((uintptr_t)p & 15u) == 0u; };
  const int vec = (L.ny % 4 == 0 && al16(a0) && al16(a1) && al16(a3) && al16(a4)) ? 1 : 0;
#define ZB_FUSED(K) \
  e = pdl_launch(K, grid, blk, sm, st, a0, a1, a2, a3, a4, to, L.nx, L.ny, idx2, vec)
#define ZB_FUSED_UP(K) \
  e = pdl_launch(K, grid, blk, sm, st, a0, a1, a2, a3, (const float*)a4, (const float*)to, a5, \
                 L.nx, L.ny, idx2, vec)
  cudaError_t e = cudaSuccess;
  if (down) {
    switch (nu) {
      case 1: ZB_FUSED((mg_down_kernel<1, TT>)); break;
      case 2: ZB_FUSED((mg_down_kernel<2, TT>)); break;
      case 3: ZB_FUSED((mg_down_kernel<3, TT>)); break;
      default: ZB_FUSED((mg_down_kernel<4, TT>)); break;
    }
  } else {
    switch (nu) {
      case 1: ZB_FUSED_UP((mg_up_kernel<1, TT>)); break;
      case 2: ZB_FUSED_UP((mg_up_kernel<2, TT>)); break;
      case 3: ZB_FUSED_UP((mg_up_kernel<3, TT>)); break;
      default: ZB_FUSED_UP((mg_up_kernel<4, TT>)); break;
    }
  }
#undef ZB_FUSED
#undef ZB_FUSED_UP
  return e == cudaSuccess ? ZB_OK : ZB_E_CUDA;
}

// 32 x 32 tiles with 256 threads when the level has a tile for every SM; else
// 16 x 16 tiles with 512 threads (four times the CTAs, two threads per staged
// cell), so that the few CTAs of a small level finish their serial phases
// sooner.  At 512^2 (256 tiles of 32^2) the large tiles win: a
// 16^2 tile stages 28^2 cells for nu = 2, three times its own
static int fused(bool down, int nu, const Level& L, float* fw, float* to, float idx2,
                 cudaStream_t st) {
  const bool big = ((L.ny + FT - 1) / FT) * ((L.nx + FT - 1) / FT) >= 148;
  if (big) return fused_level<FT>(down, nu, L, fw, to, idx2, dim3(fused_threads(FT)), st);
  return fused_level<FTS>(down, nu, L, fw, to, idx2, dim3(fused_threads(FTS)), st);
}

static int vcycle(const Plan& P, void* ws, int precond, const zb_smoother* smo, cudaStream_t st) {
  float* fw = (float*)((char*)ws + P.fbase);
  const Level& L0 = P.L[0];
  const long long n0 = (long long)L0.nx * L0.ny;
  if (precond == 0) {
    copy32_kernel<<<grid_for(n0), NT, 0, st>>>(fw + L0.f, fw + L0.xo, n0);
    return zb_launch_check();
  }
  // where a level's result lands: the fused up launch and the one-CTA kernel
  // write xo; the in-place sweeps of the coarsest level (no level fits the
  // one-CTA kernel) leave it in x
  auto result = [&](int l) -> float* {
    return (P.small0 >= P.nlev && l == P.nlev - 1) ? fw + P.L[l].x : fw + P.L[l].xo;
  };
  // fine levels: one fused launch each on the way down
  for (int l = 0; l < P.small0 && l < P.nlev - 1; ++l) {
    const Level& L = P.L[l];
    const Level& Lc = P.L[l + 1];
    const long long n = (long long)L.nx * L.ny;
    const float idx2 = 1.0f / (L.dx * L.dx);
    if (l == 0 && precond == 3) {
      zero32_kernel<<<grid_for(n), NT, 0, st>>>(fw + L.x, n);
      int rc = zb_smoother_apply(smo, fw + L.f, nullptr, fw + L.x, fw + L.cx, fw + L.cy,
                                 fw + L.r, L.nx, L.ny, (double)L.dx, 1, (void*)st);
      if (rc) return rc;
      residual32_kernel<<<grid_for(n), NT, 0, st>>>(fw + L.x, fw + L.f, fw + L.cx, fw + L.cy,
                                                    fw + L.r, L.nx, L.ny, idx2);
      restrict_kernel<<<grid_for((long long)Lc.nx * Lc.ny), NT, 0, st>>>(fw + L.r, fw + Lc.f,
                                                                          Lc.nx, Lc.ny);
    } else {
      if (const int rc = fused(true, P.nu, L, fw, fw + Lc.f, idx2, st)) return rc;
    }
  }
  if (P.small0 < P.nlev) {
    const size_t smem = coarse_smem(P);
    ZB_CUDA_TRY(pdl_launch(coarse_vcycle_kernel, dim3(1), dim3(CT), smem, st, P, fw, P.nu,
                           P.coarse_sweeps));
  } else {
    // no level fits the one-CTA kernel: sweep the coarsest level in place
    const Level& L = P.L[P.nlev - 1];
    const long long n = (long long)L.nx * L.ny;
    const float idx2 = 1.0f / (L.dx * L.dx);
    zero32_kernel<<<grid_for(n), NT, 0, st>>>(fw + L.x, n);
    for (int s = 0; s < 2 * P.coarse_sweeps; ++s) {
      const int c0 = s < P.coarse_sweeps ? 0 : 1;
      rbgs_kernel<<<grid_for(n / 2 + 1), NT, 0, st>>>(fw + L.x, fw + L.f, fw + L.cx, fw + L.cy,
                                                      fw + L.idg, L.nx, L.ny, idx2, c0);
      rbgs_kernel<<<grid_for(n / 2 + 1), NT, 0, st>>>(fw + L.x, fw + L.f, fw + L.cx, fw + L.cy,
                                                      fw + L.idg, L.nx, L.ny, idx2, 1 - c0);
    }
  }
  // fine levels on the way up: coarse correction + post-smoothing, fused
  for (int l = std::min(P.small0, P.nlev - 1) - 1; l >= 0; --l) {
    const Level& L = P.L[l];
    const Level& Lc = P.L[l + 1];
    const long long n = (long long)L.nx * L.ny;
    const float idx2 = 1.0f / (L.dx * L.dx);
    if (l == 0 && precond == 3) {
      prolong_add_kernel<<<grid_for(n), NT, 0, st>>>(result(l + 1), fw + L.x, Lc.nx, Lc.ny);
      int rc = zb_smoother_apply(smo, fw + L.f, fw + L.x, fw + L.xo, fw + L.cx, fw + L.cy,
                                 fw + L.r, L.nx, L.ny, (double)L.dx, 0, (void*)st);
      if (rc) return rc;
    } else {
      if (const int rc = fused(false, P.nu, L, fw, result(l + 1), idx2, st)) return rc;
    }
  }
  if (result(0) != fw + L0.xo)   // a single level swept in place
    copy32_kernel<<<grid_for(n0), NT, 0, st>>>(fw + L0.x, fw + L0.xo, n0);
  if (precond == 2) {
    int rc = zb_smoother_apply(smo, fw + L0.f, fw + L0.xo, fw + L0.xo, fw + L0.cx, fw + L0.cy,
                               fw + L0.r, L0.nx, L0.ny, (double)L0.dx, 0, (void*)st);
    if (rc) return rc;
  }
  return zb_launch_check();
}

}  // namespace pois
}  // namespace zb

using namespace zb;
using namespace zb::pois;

extern "C" {

size_t zb_poisson_workspace_bytes(const zb_poisson_cfg* cfg) {
  if (!valid(cfg)) return 0;
  return (size_t)make_plan(cfg).bytes;
}

int zb_poisson_layout(const zb_poisson_cfg* cfg, int64_t* out) {
  if (!valid(cfg) || !out) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  // byte offsets: r, (none), p, q (float64 Krylov vectors), scalars, the
  // V-cycle's float result on level 0 (z) and level-0 f, number of levels,
  // first one-CTA level
  out[0] = P.vr * 8;
  out[1] = -1;   // no float64 z: [5] holds z = M r
  out[2] = P.vp * 8;
  out[3] = P.vq * 8;
  out[4] = P.scal * 8;
  out[5] = P.fbase + P.L[0].xo * 4;
  out[6] = P.fbase + P.L[0].f * 4;
  out[7] = P.nlev;
  out[8] = P.small0;
  out[9] = P.fbase + P.L[0].cx * 4;
  out[10] = P.fbase + P.L[0].cy * 4;
  return ZB_OK;
}

int zb_poisson_setup(const zb_poisson_cfg* cfg, const void* h, int dtype, void* ws,
                     size_t wsb, zb_stream_t stream) {
  if (!valid(cfg) || !h || !ws || (dtype != ZB_F32 && dtype != ZB_F64)) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  if (wsb < (size_t)P.bytes) return ZB_E_ARG;
  if (P.small0 < P.nlev &&
      (coarse_smem(P) > COARSE_SMEM_MAX || P.nlev - P.small0 > CT_MAX_LEVELS))
    return ZB_E_TOO_LARGE;
  if (const int e = enable_coarse_smem()) return e;
  cudaStream_t st = (cudaStream_t)stream;
  float* fw = (float*)((char*)ws + P.fbase);
  double* dw = (double*)ws;
  const Level& L0 = P.L[0];
  const long long n0 = (long long)L0.nx * L0.ny;
  const double idx2 = 1.0 / (cfg->dx * cfg->dx);
  const float idx2f = 1.0f / (L0.dx * L0.dx);
  if (dtype == ZB_F64)
    setup0_kernel<double><<<grid_for(n0), NT, 0, st>>>(
        (const double*)h, L0.nx, L0.ny, cfg->cmin, cfg->cmax, idx2, idx2f, dw + P.cx64,
        dw + P.cy64, dw + P.dg64, fw + L0.cx, fw + L0.cy, fw + L0.idg);
  else
    setup0_kernel<float><<<grid_for(n0), NT, 0, st>>>(
        (const float*)h, L0.nx, L0.ny, cfg->cmin, cfg->cmax, idx2, idx2f, dw + P.cx64,
        dw + P.cy64, dw + P.dg64, fw + L0.cx, fw + L0.cy, fw + L0.idg);
  // levels above the one-CTA part: one launch each; the rest and the
  // coarsest inverse: one CTA
  const int l_small = std::max(1, std::min(P.small0, P.nlev));
  for (int l = 1; l < l_small; ++l) {
    const Level& L = P.L[l];
    const Level& Lf = P.L[l - 1];
    coarsen_kernel<<<grid_for((long long)L.nx * L.ny), NT, 0, st>>>(
        fw + Lf.cx, fw + Lf.cy, L.nx, L.ny, 1.0f / (L.dx * L.dx), fw + L.cx, fw + L.cy,
        fw + L.idg);
  }
  if (l_small < P.nlev || P.cinv >= 0) small_setup_kernel<<<1, ST, 0, st>>>(P, fw, l_small);
  ZB_CUDA_TRY(cudaMemsetAsync(dw + P.scal, 0, S_COUNT * sizeof(double), st));
  return zb_launch_check();
}

int zb_poisson_apply(const zb_poisson_cfg* cfg, void* ws, const double* p, double* q,
                     zb_stream_t stream) {
  if (!valid(cfg) || !ws || !p || !q) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  double* dw = (double*)ws;
  apply_dot_kernel<<<RED_BLOCKS, NT, 0, st>>>(dw + P.cx64, dw + P.cy64, p, nullptr, q, cfg->nx,
                                              cfg->ny, 1.0 / (cfg->dx * cfg->dx), dw + P.part,
                                              nullptr, nullptr, nullptr);
  return zb_launch_check();
}

int zb_poisson_vcycle(const zb_poisson_cfg* cfg, void* ws, const float* r, float* z, int precond,
                      const zb_smoother* smo, zb_stream_t stream) {
  if (!valid(cfg) || !ws || !r || !z || precond < 0 || precond > 3) return ZB_E_ARG;
  if (precond >= 2 && !smo) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  float* fw = (float*)((char*)ws + P.fbase);
  const long long n0 = (long long)cfg->nx * cfg->ny;
  copy32_kernel<<<grid_for(n0), NT, 0, st>>>(r, fw + P.L[0].f, n0);
  int rc = vcycle(P, ws, precond, smo, st);
  if (rc) return rc;
  copy32_kernel<<<grid_for(n0), NT, 0, st>>>(fw + P.L[0].xo, z, n0);
  return zb_launch_check();
}

int zb_poisson_rhs(const zb_poisson_cfg* cfg, const void* Q, int dtype, double dt, double* b,
                   zb_stream_t stream) {
  if (!valid(cfg) || !Q || !b || !(dt > 0.0)) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)cfg->nx * cfg->ny;
  const double s = 1.0 / (dt * cfg->dx);
  if (dtype == ZB_F64)
    rhs_kernel<double><<<grid_for(n), NT, 0, st>>>((const double*)Q + 2 * n,
                                                   (const double*)Q + 3 * n, cfg->nx, cfg->ny, s, b);
  else if (dtype == ZB_F32)
    rhs_kernel<float><<<grid_for(n), NT, 0, st>>>((const float*)Q + 2 * n, (const float*)Q + 3 * n,
                                                  cfg->nx, cfg->ny, s, b);
  else
    return ZB_E_ARG;
  return zb_launch_check();
}

int zb_poisson_correct(const zb_poisson_cfg* cfg, void* ws, void* Q, int dtype, const double* p,
                       double dt, zb_stream_t stream) {
  if (!valid(cfg) || !ws || !Q || !p || !(dt >= 0.0)) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  double* dw = (double*)ws;
  const long long n = (long long)cfg->nx * cfg->ny;
  if (dtype == ZB_F64)
    correct_kernel<double><<<grid_for(n), NT, 0, st>>>((double*)Q + 2 * n, (double*)Q + 3 * n,
                                                       dw + P.cx64, dw + P.cy64, p, cfg->nx,
                                                       cfg->ny, dt, 1.0 / cfg->dx);
  else if (dtype == ZB_F32)
    correct_kernel<float><<<grid_for(n), NT, 0, st>>>((float*)Q + 2 * n, (float*)Q + 3 * n,
                                                      dw + P.cx64, dw + P.cy64, p, cfg->nx,
                                                      cfg->ny, dt, 1.0 / cfg->dx);
  else
    return ZB_E_ARG;
  return zb_launch_check();
}

static int fcg_start_impl(const zb_poisson_cfg* cfg, void* ws, const double* b, double* x,
                          int precond, const zb_smoother* smo, zb_stream_t stream,
                          const LoopCtl* lc) {
  if (!valid(cfg) || !ws || !b || !x || precond < 0 || precond > 3) return ZB_E_ARG;
  if (precond >= 2 && !smo) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  double* dw = (double*)ws;
  float* fw = (float*)((char*)ws + P.fbase);
  const long long n = (long long)cfg->nx * cfg->ny;
  double* part = dw + P.part;
  double* scal = dw + P.scal;
  unsigned* ctr = counters(scal);
  ZB_CUDA_TRY(pdl_launch(residual64_kernel, dim3(RED_BLOCKS), dim3(NT), 0, st,
                         (const double*)(dw + P.cx64), (const double*)(dw + P.cy64),
                         (const double*)x, b, dw + P.vr, cfg->nx, cfg->ny,
                         1.0 / (cfg->dx * cfg->dx), part, part + RED_BLOCKS, fw + P.L[0].f, ctr,
                         scal));
  int rc = vcycle(P, ws, precond, smo, st);
  if (rc) return rc;
  const float* z32 = fw + P.L[0].xo;
  if (lc)
    ZB_CUDA_TRY(pdl_launch(p_update_cond_kernel, dim3(grid_for(n)), dim3(NT), 0, st, dw + P.vp,
                           z32, scal, n, 1, lc->h, lc->tol, lc->maxit));
  else
    ZB_CUDA_TRY(pdl_launch(p_update_kernel, dim3(grid_for(n)), dim3(NT), 0, st, dw + P.vp, z32,
                           (const double*)scal, n, 1));
  return zb_launch_check();
}

int zb_fcg_start(const zb_poisson_cfg* cfg, void* ws, const double* b, double* x, int precond,
                 const zb_smoother* smo, zb_stream_t stream) {
  return fcg_start_impl(cfg, ws, b, x, precond, smo, stream, nullptr);
}

static int fcg_iterate_impl(const zb_poisson_cfg* cfg, void* ws, double* x, int precond,
                            const zb_smoother* smo, zb_stream_t stream, const LoopCtl* lc) {
  if (!valid(cfg) || !ws || !x || precond < 0 || precond > 3) return ZB_E_ARG;
  if (precond >= 2 && !smo) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  double* dw = (double*)ws;
  float* fw = (float*)((char*)ws + P.fbase);
  const long long n = (long long)cfg->nx * cfg->ny;
  double* part = dw + P.part;
  double* scal = dw + P.scal;
  unsigned* ctr = counters(scal);
  ZB_CUDA_TRY(pdl_launch(apply_dot_kernel, dim3(RED_BLOCKS), dim3(NT), 0, st,
                         (const double*)(dw + P.cx64), (const double*)(dw + P.cy64),
                         (const double*)(dw + P.vp), (const double*)(dw + P.vr), dw + P.vq, cfg->nx,
                         cfg->ny, 1.0 / (cfg->dx * cfg->dx), part, part + RED_BLOCKS, ctr + 1,
                         scal));
  ZB_CUDA_TRY(pdl_launch(update_xr_kernel, dim3(RED_BLOCKS), dim3(NT), 0, st, x, dw + P.vr,
                         (const double*)(dw + P.vp), (const double*)(dw + P.vq), scal, n,
                         part + 2 * RED_BLOCKS, fw + P.L[0].f, ctr + 2));
  int rc = vcycle(P, ws, precond, smo, st);
  if (rc) return rc;
  const float* z32 = fw + P.L[0].xo;
  ZB_CUDA_TRY(pdl_launch(zq_kernel, dim3(RED_BLOCKS), dim3(NT), 0, st, z32,
                         (const double*)(dw + P.vq), n, part + 3 * RED_BLOCKS, ctr + 3, scal));
  if (lc)
    ZB_CUDA_TRY(pdl_launch(p_update_cond_kernel, dim3(grid_for(n)), dim3(NT), 0, st, dw + P.vp,
                           z32, scal, n, 0, lc->h, lc->tol, lc->maxit));
  else
    ZB_CUDA_TRY(pdl_launch(p_update_kernel, dim3(grid_for(n)), dim3(NT), 0, st, dw + P.vp, z32,
                           (const double*)scal, n, 0));
  return zb_launch_check();
}

int zb_fcg_iterate(const zb_poisson_cfg* cfg, void* ws, double* x, int precond,
                   const zb_smoother* smo, zb_stream_t stream) {
  return fcg_iterate_impl(cfg, ws, x, precond, smo, stream, nullptr);
}


// A whole FCG solve as one CUDA graph: the start, then a conditional WHILE
// node whose body is one iteration plus the loop-control kernel.  One launch
// runs to convergence (or maxit) with no host round trip; the iteration count
// lands at scalar index 8 and the relative residual at index 7.
struct zb_fcg_graph {
  cudaGraphExec_t exec;
  cudaGraph_t graph;
};

int zb_fcg_graph_create(const zb_poisson_cfg* cfg, void* ws, const double* b, double* x,
                        int precond, const zb_smoother* smo, double tol, int maxit,
                        zb_fcg_graph** out, zb_stream_t stream) {
  if (!valid(cfg) || !ws || !b || !x || !out || precond < 0 || precond > 3 || maxit < 1 ||
      !(tol >= 0.0))
    return ZB_E_ARG;
  if (precond >= 2 && !smo) return ZB_E_ARG;
  *out = nullptr;
  (void)stream;   // capture runs on private streams; nothing executes here
  const Plan P = make_plan(cfg);
  cudaStream_t st = nullptr, body = nullptr;
  ZB_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(st);
    return ZB_E_CUDA;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  int rc = ZB_OK;
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) { cudaStreamDestroy(body); cudaStreamDestroy(st); return ZB_E_CUDA; }
  do {
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr) != cudaSuccess) { rc = ZB_E_CUDA; break; }
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, g, 0u, cudaGraphCondAssignDefault) != cudaSuccess) { rc = ZB_E_CUDA; break; }
    const LoopCtl lc = {h, tol, maxit};
    if ((rc = fcg_start_impl(cfg, ws, b, x, precond, smo, (void*)st, &lc))) break;
    if (cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps) != cudaSuccess) { rc = ZB_E_CUDA; break; }
    cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, g, deps, ndeps, &np) != cudaSuccess) { rc = ZB_E_CUDA; break; }
    cudaGraph_t bg = np.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(body, bg, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess) { rc = ZB_E_CUDA; break; }
    int rb = fcg_iterate_impl(cfg, ws, x, precond, smo, (void*)body, &lc);
    cudaGraph_t bg2 = nullptr;
    const cudaError_t eb = cudaStreamEndCapture(body, &bg2);
    if (rb) { rc = rb; break; }
    if (eb != cudaSuccess) { rc = ZB_E_CUDA; break; }
    if (cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) { rc = ZB_E_CUDA; break; }
  } while (0);
  cudaGraph_t gout = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(st, &gout);
  cudaStreamDestroy(body);
  cudaStreamDestroy(st);
  if (rc == ZB_OK && ee != cudaSuccess) rc = ZB_E_CUDA;
  if (rc != ZB_OK) {
    if (gout) cudaGraphDestroy(gout);
    cudaGetLastError();
    return rc;
  }
  if (cudaGraphInstantiate(&ex, gout, 0) != cudaSuccess) {
    cudaGraphDestroy(gout);
    cudaGetLastError();
    return ZB_E_CUDA;
  }
  zb_fcg_graph* G = new zb_fcg_graph;
  G->exec = ex;
  G->graph = gout;
  *out = G;
  return ZB_OK;
}

int zb_fcg_graph_launch(zb_fcg_graph* G, zb_stream_t stream) {
  if (!G) return ZB_E_ARG;
  ZB_CUDA_TRY(cudaGraphLaunch(G->exec, (cudaStream_t)stream));
  return ZB_OK;
}

void zb_fcg_graph_destroy(zb_fcg_graph* G) {
  if (!G) return;
  cudaGraphExecDestroy(G->exec);
  cudaGraphDestroy(G->graph);
  delete G;
}


// Synchronous convenience solve for C callers: FCG from the x given until
// |r| / |b| <= tol or maxit iterations, reading the relative residual after
// each iteration (one stream synchronisation per iteration).
int zb_poisson_solve(const zb_poisson_cfg* cfg, void* ws, const double* b, double* x, double tol,
                     int maxit, int precond, const zb_smoother* smo, int* out_iters,
                     double* out_rel, zb_stream_t stream) {
  if (!valid(cfg) || !ws || !b || !x || maxit < 0 || !(tol >= 0.0)) return ZB_E_ARG;
  const Plan P = make_plan(cfg);
  cudaStream_t st = (cudaStream_t)stream;
  const double* rel_dev = (const double*)ws + P.scal + S_REL;
  int rc = zb_fcg_start(cfg, ws, b, x, precond, smo, stream);
  if (rc) return rc;
  double rel = 0.0;
  int it = 0;
  for (;;) {
    ZB_CUDA_TRY(cudaMemcpyAsync(&rel, rel_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
    ZB_CUDA_TRY(cudaStreamSynchronize(st));
    if (!(rel > tol) || it >= maxit) break;
    if ((rc = zb_fcg_iterate(cfg, ws, x, precond, smo, stream))) return rc;
    ++it;
  }
  if (out_iters) *out_iters = it;
  if (out_rel) *out_rel = rel;
  return rel <= tol ? ZB_OK : ZB_E_NOT_CONVERGED;
}

}  // extern "C"
