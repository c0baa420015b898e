// Triangle mesh preparation on the GPU (sm_100a): from vertices and
// triangles to the device arrays of zb_tri_mesh -- the work the reference does
// on the host when it turns zoomy_core's LSQMesh into MeshJAX arrays
// (zoomy_jax/mesh/mesh.py:123-264) and derives the runtime index sets
// (zoomy_jax/fvm/solver2/context.py:99-163: owner / neighbour per face,
// interior / boundary split, inradius, least-squares stencils).
//
//   phase 1 (zb_trimesh_match)
//     tm_insert_kernel   one thread per cell: counter-clockwise orientation,
//                        area, centroid, inradius 2 area / perimeter; its three
//                        half-edges go into an open-addressing hash keyed by
//                        the vertex pair (splitmix64 finaliser, linear probing,
//                        bounded), two half-edge slots per key
//     tm_link_kernel     one thread per cell: each half-edge's twin (or none:
//                        a boundary face); the lower cell index owns a shared
//                        face, a boundary face belongs to its cell; per-cell
//                        counts of owned faces and boundary faces
//     scan (3 kernels)   exclusive prefix sums of the two counts: the face and
//                        boundary-face numbers are (owner cell, local edge)
//                        order -- deterministic whatever order the hash
//                        inserts ran in
//   phase 2 (zb_trimesh_fill)
//     tm_face_kernel     one thread per cell, over its owned faces: owner,
//                        neighbour or -1 - boundary number, unit normal out of
//                        the owner, length, centre offsets, CFL inradius, and
//                        for boundary faces the kind of the side its normal
//                        faces (left / right / bottom / top)
//     tm_cell_kernel     one thread per cell: its three faces in increasing
//                        face number with the side flag, face-centre offsets,
//                        least-squares stencil (neighbour centroid, or the
//                        ghost at twice the face-centre offset, counted for
//                        derivative d only where the normal has a d component)
//                        and the weights of the 2x2 normal equations
// Geometry is float64 throughout and is written in the state precision
// (face_inr stays float64).  A non-manifold edge (three triangles), a vertex
// index out of range or a zero-area triangle sets an error flag that the host
// turns into ZB_E_ARG.
#include <cstring>
#include <algorithm>

#include "common.cuh"

namespace zb {
namespace tmp {

constexpr int NT = 256;
constexpr int SCAN_NT = 1024;
constexpr unsigned long long EMPTY = ~0ull;
enum { ERR_VERTEX = 1, ERR_NONMANIFOLD = 2, ERR_TABLE = 4, ERR_DEGENERATE = 8 };

// splitmix64 output function (Steele, Lea and Flood 2014): spreads the packed
// vertex pair over the table
__device__ __forceinline__ unsigned long long mix64(unsigned long long k) {
  k ^= k >> 30;
  k *= 0xbf58476d1ce4e5b9ull;
  k ^= k >> 27;
  k *= 0x94d049bb133111ebull;
  k ^= k >> 31;
  return k;
}

// scratch layout (every block 256-byte aligned)
struct Layout {
  size_t keys, he0, he1, tf, slot, nbr, cnt, base, bsum, xc, area, inr, hface, hbnum, flags;
  size_t total;
  int hash_bits, nblk;
};

static size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

static Layout layout(long long C) {
  Layout L;
  int hb = 4;
  while ((1ll << hb) < 3 * C) ++hb;       // >= 3C slots for ~1.5C keys
  L.hash_bits = hb;
  const size_t S = size_t(1) << hb;
  L.nblk = (int)((C + SCAN_NT - 1) / SCAN_NT);
  size_t o = 0;
  auto take = [&](size_t bytes) { const size_t at = o; o += a256(bytes); return at; };
  L.keys = take(S * 8);
  L.he0 = take(S * 4);
  L.he1 = take(S * 4);
  L.tf = take(size_t(3 * C) * 4);
  L.slot = take(size_t(3 * C) * 4);
  L.nbr = take(size_t(3 * C) * 4);
  L.cnt = take(size_t(C) * 8);
  L.base = take(size_t(C) * 8);
  L.bsum = take(size_t(L.nblk) * 8);
  L.xc = take(size_t(C) * 16);
  L.area = take(size_t(C) * 8);
  L.inr = take(size_t(C) * 8);
  L.hface = take(size_t(3 * C) * 4);
  L.hbnum = take(size_t(3 * C) * 4);
  L.flags = take(64);                     // int err; int2 totals
  L.total = o;
  return L;
}

__global__ void __launch_bounds__(NT)
tm_insert_kernel(const double* __restrict__ P, int nv, const int* __restrict__ T, int C,
                 int* __restrict__ Tf, double2* __restrict__ xc, double* __restrict__ area,
                 double* __restrict__ inr, unsigned long long* keys, int* he0, int* he1,
                 int* __restrict__ slot, unsigned long long mask, int* err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int v[3] = {T[3 * c], T[3 * c + 1], T[3 * c + 2]};
  if (v[0] < 0 || v[0] >= nv || v[1] < 0 || v[1] >= nv || v[2] < 0 || v[2] >= nv ||
      v[0] == v[1] || v[1] == v[2] || v[0] == v[2]) {
    atomicOr(err, ERR_VERTEX);
    v[0] = v[1] = v[2] = 0;
  }
  double2 p[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) p[k] = make_double2(P[2 * v[k]], P[2 * v[k] + 1]);
  const double cross = (p[1].x - p[0].x) * (p[2].y - p[0].y) - (p[1].y - p[0].y) * (p[2].x - p[0].x);
  if (cross < 0.0) {
    int tv = v[1]; v[1] = v[2]; v[2] = tv;
    double2 tp = p[1]; p[1] = p[2]; p[2] = tp;
  }
  if (cross == 0.0 && v[0] != v[1]) atomicOr(err, ERR_DEGENERATE);
  const double a = 0.5 * fabs(cross);
  const double per = hypot(p[1].x - p[0].x, p[1].y - p[0].y) +
                     hypot(p[2].x - p[1].x, p[2].y - p[1].y) +
                     hypot(p[0].x - p[2].x, p[0].y - p[2].y);
  area[c] = a;
  inr[c] = 2.0 * a / per;
  xc[c] = make_double2((p[0].x + p[1].x + p[2].x) / 3.0, (p[0].y + p[1].y + p[2].y) / 3.0);
#pragma unroll
  for (int k = 0; k < 3; ++k) Tf[3 * c + k] = v[k];
  if (v[0] == v[1]) return;               // invalid cell: flagged above
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int va = v[k], vb = v[(k + 1) % 3];
    const unsigned long long key =
        ((unsigned long long)min(va, vb) << 32) | (unsigned long long)max(va, vb);
    const int he = 3 * c + k;
    unsigned long long h = mix64(key) & mask;
    bool placed = false;
    for (unsigned long long probe = 0; probe <= mask; ++probe) {
      const unsigned long long prev = atomicCAS(&keys[h], EMPTY, key);
      if (prev == EMPTY || prev == key) {
        if (atomicCAS(&he0[h], -1, he) != -1 && atomicCAS(&he1[h], -1, he) != -1)
          atomicOr(err, ERR_NONMANIFOLD);
        slot[he] = (int)h;
        placed = true;
        break;
      }
      h = (h + 1) & mask;
    }
    if (!placed) {
      atomicOr(err, ERR_TABLE);
      slot[he] = -1;
    }
  }
}

__device__ __forceinline__ bool owns(int he, int other) {
  return other < 0 || other / 3 > he / 3;
}

__global__ void __launch_bounds__(NT)
tm_link_kernel(int C, const int* __restrict__ he0, const int* __restrict__ he1,
               const int* __restrict__ slot, int* __restrict__ nbr, int2* __restrict__ cnt,
               int* err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int own = 0, bnd = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int he = 3 * c + k;
    const int h = slot[he];
    int other = -1;
    if (h >= 0) {
      const int a = he0[h], b = he1[h];
      other = a == he ? b : a;
    }
    if (other >= 0 && other / 3 == c) {   // a triangle meeting itself
      atomicOr(err, ERR_DEGENERATE);
      other = -1;
    }
    nbr[he] = other;
    own += owns(he, other) ? 1 : 0;
    bnd += other < 0 ? 1 : 0;
  }
  cnt[c] = make_int2(own, bnd);
}

// exclusive scan of int2 counts: block sums, one-CTA scan of the block sums,
// block-local scan plus offset
__device__ __forceinline__ int2 block_scan_excl(int2 v, int2* sh, int2* total) {
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int o = 1; o < SCAN_NT; o <<= 1) {
    int2 add = make_int2(0, 0);
    if (t >= o) add = sh[t - o];
    __syncthreads();
    sh[t].x += add.x;
    sh[t].y += add.y;
    __syncthreads();
  }
  const int2 incl = sh[t];
  *total = sh[SCAN_NT - 1];
  __syncthreads();
  return make_int2(incl.x - v.x, incl.y - v.y);
}

__global__ void __launch_bounds__(SCAN_NT)
tm_scan_blocks(const int2* __restrict__ cnt, int C, int2* __restrict__ bsum) {
  __shared__ int2 sh[SCAN_NT];
  const int i = blockIdx.x * SCAN_NT + threadIdx.x;
  const int2 v = i < C ? cnt[i] : make_int2(0, 0);
  int2 tot;
  block_scan_excl(v, sh, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_NT)
tm_scan_sums(int2* __restrict__ bsum, int nblk, int2* __restrict__ totals) {
  __shared__ int2 sh[SCAN_NT];
  int2 carry = make_int2(0, 0);
  for (int b0 = 0; b0 < nblk; b0 += SCAN_NT) {
    const int i = b0 + threadIdx.x;
    const int2 v = i < nblk ? bsum[i] : make_int2(0, 0);
    int2 tot;
    const int2 ex = block_scan_excl(v, sh, &tot);
    if (i < nblk) bsum[i] = make_int2(ex.x + carry.x, ex.y + carry.y);
    carry.x += tot.x;
    carry.y += tot.y;
  }
  if (threadIdx.x == 0) *totals = carry;
}

__global__ void __launch_bounds__(SCAN_NT)
tm_scan_apply(const int2* __restrict__ cnt, int C, const int2* __restrict__ bsum,
              int2* __restrict__ base) {
  __shared__ int2 sh[SCAN_NT];
  const int i = blockIdx.x * SCAN_NT + threadIdx.x;
  const int2 v = i < C ? cnt[i] : make_int2(0, 0);
  int2 tot;
  const int2 ex = block_scan_excl(v, sh, &tot);
  const int2 off = bsum[blockIdx.x];
  if (i < C) base[i] = make_int2(ex.x + off.x, ex.y + off.y);
}

template <typename T>
struct Out {
  int* lsq_idx;
  T* lsq_wx;
  T* lsq_wy;
  T* cf_rx;
  T* cf_ry;
  int* cell_face;
  T* cell_inv_area;
  int* face_a;
  int* face_b;
  T* face_nx;
  T* face_ny;
  T* face_len;
  T* face_rax;
  T* face_ray;
  T* face_rbx;
  T* face_rby;
  double* face_inr;
  int* bf_kind;
  T* bf_nx;
  T* bf_ny;
};

template <typename T>
__global__ void __launch_bounds__(NT)
tm_face_kernel(const double* __restrict__ P, int C, const int* __restrict__ Tf,
               const int* __restrict__ nbr, const int2* __restrict__ base,
               const double2* __restrict__ xc, const double* __restrict__ inr,
               int4 kinds, int* __restrict__ hface, int* __restrict__ hbnum, Out<T> o) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  int f = base[c].x, bn = base[c].y;
  const double2 xa = xc[c];
  const int kind[4] = {kinds.x, kinds.y, kinds.z, kinds.w};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int he = 3 * c + k;
    const int other = nbr[he];
    if (!owns(he, other)) continue;
    const int va = Tf[3 * c + k], vb = Tf[3 * c + (k + 1) % 3];
    const double ax = P[2 * va], ay = P[2 * va + 1], bx = P[2 * vb], by = P[2 * vb + 1];
    const double tx = bx - ax, ty = by - ay;
    const double L = hypot(tx, ty);
    const double nx = ty / L, ny = -tx / L;
    const double fx = 0.5 * (ax + bx), fy = 0.5 * (ay + by);
    const double rax = fx - xa.x, ray = fy - xa.y;
    double rbx = rax, rby = ray, ir = inr[c];
    o.face_a[f] = c;
    if (other >= 0) {
      const int cb = other / 3;
      const double2 xb = xc[cb];
      rbx = fx - xb.x;
      rby = fy - xb.y;
      ir = fmin(ir, inr[cb]);
      o.face_b[f] = cb;
      hface[other] = 2 * f + 1;
      hbnum[other] = -1;
      hbnum[he] = -1;
    } else {
      // the side its normal faces: left, right, bottom, top
      const int tag = nx < -0.5 ? 0 : (nx > 0.5 ? 1 : (ny < 0.0 ? 2 : 3));
      o.face_b[f] = -(bn + 1);
      o.bf_kind[bn] = kind[tag];
      o.bf_nx[bn] = (T)nx;
      o.bf_ny[bn] = (T)ny;
      hbnum[he] = bn;
      ++bn;
    }
    hface[he] = 2 * f;
    o.face_nx[f] = (T)nx;
    o.face_ny[f] = (T)ny;
    o.face_len[f] = (T)L;
    o.face_rax[f] = (T)rax;
    o.face_ray[f] = (T)ray;
    o.face_rbx[f] = (T)rbx;
    o.face_rby[f] = (T)rby;
    o.face_inr[f] = ir;
    ++f;
  }
}

template <typename T>
__global__ void __launch_bounds__(NT)
tm_cell_kernel(const double* __restrict__ P, int C, const int* __restrict__ Tf,
               const int* __restrict__ nbr, const double2* __restrict__ xc,
               const double* __restrict__ area, const int* __restrict__ hface,
               const int* __restrict__ hbnum, Out<T> o) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  // the three half-edges in increasing face number
  int ks[3] = {0, 1, 2};
  int hf[3] = {hface[3 * c], hface[3 * c + 1], hface[3 * c + 2]};
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2 - i; ++j)
      if ((hf[j] >> 1) > (hf[j + 1] >> 1)) {
        int t = hf[j]; hf[j] = hf[j + 1]; hf[j + 1] = t;
        t = ks[j]; ks[j] = ks[j + 1]; ks[j + 1] = t;
      }
  const double2 x0 = xc[c];
  double mx[3], my[3];
  bool ux[3], uy[3];
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int k = ks[s], he = 3 * c + k;
    const int va = Tf[3 * c + k], vb = Tf[3 * c + (k + 1) % 3];
    const double ax = P[2 * va], ay = P[2 * va + 1], bx = P[2 * vb], by = P[2 * vb + 1];
    const double fx = 0.5 * (ax + bx), fy = 0.5 * (ay + by);
    const double rx = fx - x0.x, ry = fy - x0.y;
    o.cell_face[s * C + c] = hf[s];
    o.cf_rx[s * C + c] = (T)rx;
    o.cf_ry[s * C + c] = (T)ry;
    const int other = nbr[he];
    if (other >= 0) {
      const double2 xb = xc[other / 3];
      mx[s] = xb.x - x0.x;
      my[s] = xb.y - x0.y;
      ux[s] = uy[s] = true;
      o.lsq_idx[s * C + c] = other / 3;
    } else {
      // ghost at twice the face-centre offset; it enters derivative d only
      // where the face normal has a d component
      const double tx = bx - ax, ty = by - ay;
      const double L = hypot(tx, ty);
      mx[s] = 2.0 * rx;
      my[s] = 2.0 * ry;
      ux[s] = fabs(ty / L) > 1e-12;
      uy[s] = fabs(-tx / L) > 1e-12;
      o.lsq_idx[s * C + c] = -(hbnum[he] + 1);
    }
  }
  // per direction: normal matrix of the used offsets, its inverse, weights
#pragma unroll
  for (int d = 0; d < 2; ++d) {
    double sxx = 0.0, sxy = 0.0, syy = 0.0;
    double px[3], py[3];
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const bool u = d == 0 ? ux[s] : uy[s];
      px[s] = u ? mx[s] : 0.0;
      py[s] = u ? my[s] : 0.0;
      sxx += px[s] * px[s];
      sxy += px[s] * py[s];
      syy += py[s] * py[s];
    }
    const double det = sxx * syy - sxy * sxy;
    const double i0 = d == 0 ? syy / det : -sxy / det;
    const double i1 = d == 0 ? -sxy / det : sxx / det;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const double w = i0 * px[s] + i1 * py[s];
      if (d == 0) o.lsq_wx[s * C + c] = (T)w;
      else o.lsq_wy[s * C + c] = (T)w;
    }
  }
  o.cell_inv_area[c] = (T)(1.0 / area[c]);
}

template <typename T>
static Out<T> out_of(const zb_tri_mesh* m) {
  Out<T> o;
  o.lsq_idx = const_cast<int*>(m->lsq_idx);
  o.lsq_wx = (T*)m->lsq_wx;
  o.lsq_wy = (T*)m->lsq_wy;
  o.cf_rx = (T*)m->cf_rx;
  o.cf_ry = (T*)m->cf_ry;
  o.cell_face = const_cast<int*>(m->cell_face);
  o.cell_inv_area = (T*)m->cell_inv_area;
  o.face_a = const_cast<int*>(m->face_a);
  o.face_b = const_cast<int*>(m->face_b);
  o.face_nx = (T*)m->face_nx;
  o.face_ny = (T*)m->face_ny;
  o.face_len = (T*)m->face_len;
  o.face_rax = (T*)m->face_rax;
  o.face_ray = (T*)m->face_ray;
  o.face_rbx = (T*)m->face_rbx;
  o.face_rby = (T*)m->face_rby;
  o.face_inr = const_cast<double*>(m->face_inr);
  o.bf_kind = const_cast<int*>(m->bf_kind);
  o.bf_nx = (T*)m->bf_nx;
  o.bf_ny = (T*)m->bf_ny;
  return o;
}

}  // namespace tmp
}  // namespace zb

using namespace zb;
using namespace zb::tmp;

extern "C" {

size_t zb_trimesh_scratch_bytes(int32_t n_cells) {
  if (n_cells < 1 || (long long)n_cells * 3 >= (1ll << 31)) return 0;
  return layout(n_cells).total;
}

int zb_trimesh_match(const double* P, int32_t n_vert, const int32_t* T, int32_t n_cells,
                     void* scratch, size_t scratch_bytes, int32_t* n_faces, int32_t* n_bf,
                     zb_stream_t stream) {
  if (!P || !T || !scratch || !n_faces || !n_bf || n_vert < 3 || n_cells < 1) return ZB_E_ARG;
  if ((long long)n_cells * 3 >= (1ll << 31)) return ZB_E_TOO_LARGE;
  const Layout L = layout(n_cells);
  if (scratch_bytes < L.total) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  char* s = (char*)scratch;
  const size_t S = size_t(1) << L.hash_bits;
  ZB_CUDA_TRY(cudaMemsetAsync(s + L.keys, 0xFF, S * 8, st));
  ZB_CUDA_TRY(cudaMemsetAsync(s + L.he0, 0xFF, S * 4, st));
  ZB_CUDA_TRY(cudaMemsetAsync(s + L.he1, 0xFF, S * 4, st));
  ZB_CUDA_TRY(cudaMemsetAsync(s + L.flags, 0, 64, st));
  int* err = (int*)(s + L.flags);
  int2* totals = (int2*)(s + L.flags + 8);
  const int C = n_cells;
  const int g = (C + NT - 1) / NT;
  tm_insert_kernel<<<g, NT, 0, st>>>(P, n_vert, T, C, (int*)(s + L.tf), (double2*)(s + L.xc),
                                     (double*)(s + L.area), (double*)(s + L.inr),
                                     (unsigned long long*)(s + L.keys), (int*)(s + L.he0),
                                     (int*)(s + L.he1), (int*)(s + L.slot), S - 1, err);
  tm_link_kernel<<<g, NT, 0, st>>>(C, (const int*)(s + L.he0), (const int*)(s + L.he1),
                                   (const int*)(s + L.slot), (int*)(s + L.nbr),
                                   (int2*)(s + L.cnt), err);
  tm_scan_blocks<<<L.nblk, SCAN_NT, 0, st>>>((const int2*)(s + L.cnt), C, (int2*)(s + L.bsum));
  tm_scan_sums<<<1, SCAN_NT, 0, st>>>((int2*)(s + L.bsum), L.nblk, totals);
  tm_scan_apply<<<L.nblk, SCAN_NT, 0, st>>>((const int2*)(s + L.cnt), C,
                                            (const int2*)(s + L.bsum), (int2*)(s + L.base));
  ZB_CUDA_TRY(cudaGetLastError());
  int host[4];
  ZB_CUDA_TRY(cudaMemcpyAsync(host, s + L.flags, 16, cudaMemcpyDeviceToHost, st));
  ZB_CUDA_TRY(cudaStreamSynchronize(st));
  if (host[0] != 0) return ZB_E_ARG;
  *n_faces = host[2];
  *n_bf = host[3];
  return ZB_OK;
}

int zb_trimesh_fill(const double* P, int32_t n_cells, const int32_t* bc_kind_by_side,
                    int32_t dtype, const void* scratch, size_t scratch_bytes,
                    zb_tri_mesh* mesh, zb_stream_t stream) {
  if (!P || !bc_kind_by_side || !scratch || !mesh || n_cells < 1) return ZB_E_ARG;
  if (dtype != ZB_F32 && dtype != ZB_F64) return ZB_E_ARG;
  if (mesh->n_cells != n_cells) return ZB_E_ARG;
  const Layout L = layout(n_cells);
  if (scratch_bytes < L.total) return ZB_E_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  const char* s = (const char*)scratch;
  int* hface = (int*)(s + L.hface);
  int* hbnum = (int*)(s + L.hbnum);
  const int C = n_cells;
  const int g = (C + NT - 1) / NT;
  const int4 kinds = make_int4(bc_kind_by_side[0], bc_kind_by_side[1], bc_kind_by_side[2],
                               bc_kind_by_side[3]);
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const Out<T> o = out_of<T>(mesh);
    tm_face_kernel<T><<<g, NT, 0, st>>>(P, C, (const int*)(s + L.tf), (const int*)(s + L.nbr),
                                        (const int2*)(s + L.base), (const double2*)(s + L.xc),
                                        (const double*)(s + L.inr), kinds, hface, hbnum, o);
    tm_cell_kernel<T><<<g, NT, 0, st>>>(P, C, (const int*)(s + L.tf), (const int*)(s + L.nbr),
                                        (const double2*)(s + L.xc), (const double*)(s + L.area),
                                        hface, hbnum, o);
  };
  if (dtype == ZB_F64) run(double());
  else run(float());
  return zb_launch_check();
}

}  // extern "C"
