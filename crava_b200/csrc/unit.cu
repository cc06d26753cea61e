// unit.cu -- the fused posterior unit in three kernels per call:
//
//  k_plane_fwd  one thread-block cluster per (grid, z-plane).  Each CTA of
//               the cluster loads a band of rows, transforms them along x
//               (R2C), and scatters the half-spectrum values into the shared
//               memory of the CTA that owns their kx column pairs
//               (distributed shared memory); after a cluster barrier each CTA
//               transforms its columns along y and writes them to the
//               column-pair workspace W (two kx columns per (ky, pair) tile,
//               contiguous in z).
//  k_zsolve     one CTA per (ky, pair) tile: loads the tile of every input
//               grid (3 means, ntheta stacks, 6 prior covariances, noise
//               correlation), transforms along z, runs the per-bin posterior
//               solve on every kz, inverse-transforms the 3 + ntheta + 6
//               outputs along z and writes them back.
//  k_plane_inv  the mirror of k_plane_fwd: y inverse on column owners,
//               scatter to row owners, x C2R, scaling (and an optional
//               real addend), write to the reference layout.
//
// Every grid is read once and written once per kernel, so one unit moves
// 3 (19 + 2 ntheta) grids of HBM traffic: the reference's 29 transforms
// plus the solve (src/crava.cpp:175-190, 1003, 1012, 1042-1151, 1181-1206,
// 218) at one read and one write per transform.
#include <cooperative_groups.h>

#include <algorithm>

#include "fft_core.cuh"
#include "solve_bin.cuh"
#include "unit.cuh"

namespace cg = cooperative_groups;

namespace crava {

namespace {

constexpr int kThreads = 384;       // z transform + solve
constexpr int kPlaneThreads = 512;  // plane kernels (2 CTAs per SM)

struct PlaneArgs {
  int nxp, nyp, nzp, cnxp, rnxp, hx, even, NP, CS, R, PP, PR, PC, SA, SB, SC;
  int nitems;  // (grid, z-plane) items; each cluster loops over items
  FastDiv f_nzp;
  FastDiv f_hx, f_hx1, f_cnxp, f_nyp, f_PP, f_R;
  RadixList rx, ry;
  const float2 *twx, *twy, *post;
  const float *src_r[kMaxUnitGrids];
  float2 *w[kMaxUnitGrids];
  float *dst_r[kMaxUnitGrids];
  const float *add[kMaxUnitGrids];
  float scale[kMaxUnitGrids];
};

// Shared-memory layouts (float2 units, odd pitches keep the element-major
// accesses conflict-free):
//   row band   [m][r]  pitch PR : element m of row r of this CTA's rows
//   columns    [ky][c] pitch PC : column c (kx = 2 p0 + c) of this CTA
// Buffers: A (SA) and B (SB) carry the x transform, Cb (SC) receives the
// column values from every CTA of the cluster and, with A, the y transform.

// ------------------------------------------------------------------ forward
__global__ void __launch_bounds__(kPlaneThreads, 2) k_plane_fwd(const __grid_constant__ PlaneArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 sm4[];
  float2 *A = reinterpret_cast<float2 *>(sm4), *B = A + a.SA, *Cb = B + a.SB;
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, nth = blockDim.x;
  const int hx = a.hx, nyp = a.nyp, cnxp = a.cnxp, PR = a.PR, PC = a.PC;
  const int p0 = rank * a.PP;
  const int np_ = max(0, min(a.PP, a.NP - p0));
  const int ncol = 2 * np_;
  const int ncl = gridDim.x / a.CS;
  for (int item = blockIdx.x / a.CS; item < a.nitems; item += ncl) {
  const int gi = (int)fdiv((uint32_t)item, a.f_nzp);
  const int z = item - gi * a.nzp;
  __syncthreads();  // this CTA is done with the previous item's buffers
  // the second column of an odd last pair (kx = cnxp) is zero
  if (2 * p0 + ncol > cnxp)
    for (int ky = tid; ky < nyp; ky += nth) Cb[ky * PC + (cnxp - 2 * p0)] = make_float2(0.f, 0.f);
  cl.sync();  // every CTA of the cluster is running before remote writes

  const int y0 = rank * a.R;
  const int nr = max(0, min(a.R, nyp - y0));
  const float *plane = a.src_r[gi] + (long long)z * nyp * a.rnxp;
  const float sc = a.scale[gi];
  // every element copy of the band in flight at once (the scale is applied
  // after the transform, which is linear)
  for (int idx = tid; idx < nr * hx; idx += nth) {
    const int r = (int)fdiv((uint32_t)idx, a.f_hx), m = idx - r * hx;
    const float *row = plane + (long long)(y0 + r) * a.rnxp;
    if (a.even) cp_async8(A + m * PR + r, reinterpret_cast<const float2 *>(row) + m);
    else A[m * PR + r] = make_float2(__ldg(row + m), 0.f);
  }
  cp_async_wait_all();
  __syncthreads();
  const float2 *res = A;
  if (nr > 0) res = stockham<-1, true>(A, 1, PR, B, 1, PR, a.rx, a.twx, nr) ? B : A;
  // split to the half spectrum; scatter each value to the owner of its column
  for (int idx = tid; idx < nr * cnxp; idx += nth) {
    const int r = (int)fdiv((uint32_t)idx, a.f_cnxp), k = idx - r * cnxp;
    float2 X;
    if (a.even) {
      float2 zk = res[(k == hx ? 0 : k) * PR + r];
      float2 zm = res[(k == 0 ? 0 : hx - k) * PR + r];
      zm.y = -zm.y;
      float2 e = cscale(cadd(zk, zm), 0.5f);
      float2 d = csub(zk, zm);
      float2 o = make_float2(0.5f * d.y, -0.5f * d.x);
      X = cadd(e, cmul(__ldg(a.post + k), o));
    } else {
      X = res[k * PR + r];
    }
    X = cscale(X, sc);
    const int o = (int)fdiv((uint32_t)(k >> 1), a.f_PP);
    const int c = k - 2 * a.PP * o;
    float2 *dst = cl.map_shared_rank(Cb, o);
    dst[(y0 + r) * PC + c] = X;
  }
  cl.sync();
  if (ncol > 0) {
    res = stockham<-1, true>(Cb, 1, PC, A, 1, PC, a.ry, a.twy, ncol) ? A : Cb;
    float2 *w = a.w[gi];
    for (int idx = tid; idx < a.PP * nyp; idx += nth) {
      const int ky = (int)fdiv((uint32_t)idx, a.f_PP), pl = idx - ky * a.PP;
      if (pl >= np_) continue;
      const float2 v0 = res[ky * PC + 2 * pl], v1 = res[ky * PC + 2 * pl + 1];
      const long long off = (((long long)ky * a.NP + p0 + pl) * a.nzp + z) * 2;
      *reinterpret_cast<float4 *>(w + off) = make_float4(v0.x, v0.y, v1.x, v1.y);
    }
  }
  }  // items (the next item starts with a cluster barrier)
}

// ------------------------------------------------------------------ inverse
__global__ void __launch_bounds__(kPlaneThreads, 2) k_plane_inv(const __grid_constant__ PlaneArgs a) {
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ float4 sm4[];
  float2 *A = reinterpret_cast<float2 *>(sm4), *B = A + a.SA, *Cb = B + a.SB;
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, nth = blockDim.x;
  const int hx = a.hx, nyp = a.nyp, cnxp = a.cnxp, PR = a.PR, PC = a.PC;
  const int p0 = rank * a.PP;
  const int np_ = max(0, min(a.PP, a.NP - p0));
  const int ncol = 2 * np_;
  const int ncl = gridDim.x / a.CS;
  for (int item = blockIdx.x / a.CS; item < a.nitems; item += ncl) {
  const int gi = (int)fdiv((uint32_t)item, a.f_nzp);
  const int z = item - gi * a.nzp;
  cl.sync();  // every CTA of the cluster is running (and done with the last item)

  const float2 *w = a.w[gi];
  for (int idx = tid; idx < a.PP * nyp; idx += nth) {
    const int ky = (int)fdiv((uint32_t)idx, a.f_PP), pl = idx - ky * a.PP;
    if (pl >= np_) continue;
    const long long off = (((long long)ky * a.NP + p0 + pl) * a.nzp + z) * 2;
    cp_async8(Cb + ky * PC + 2 * pl, w + off);
    cp_async8(Cb + ky * PC + 2 * pl + 1, w + off + 1);
  }
  cp_async_wait_all();
  __syncthreads();
  const float2 *res = Cb;
  if (ncol > 0) res = stockham<1, true>(Cb, 1, PC, A, 1, PC, a.ry, a.twy, ncol) ? A : Cb;
  // scatter my columns (kx < cnxp) to the CTAs owning their rows
  const int ncv = max(0, min(ncol, cnxp - 2 * p0));
  for (int idx = tid; idx < ncv * nyp; idx += nth) {
    const int c = (int)fdiv((uint32_t)idx, a.f_nyp), ky = idx - c * nyp;
    const int o = (int)fdiv((uint32_t)ky, a.f_R), r = ky - o * a.R;
    float2 *dst = cl.map_shared_rank(B, o);
    dst[(2 * p0 + c) * PR + r] = res[ky * PC + c];
  }
  cl.sync();
  const int y0 = rank * a.R;
  const int nr = max(0, min(a.R, nyp - y0));
  for (int idx = tid; idx < a.R * hx; idx += nth) {
    const int k = (int)fdiv((uint32_t)idx, a.f_R), r = idx - k * a.R;
    if (r >= nr) continue;
    float2 v;
    if (a.even) {
      // Z'[k] = (X_k + conj X_{h-k}) + i W^{-k} (X_k - conj X_{h-k}); the
      // imaginary parts of DC and Nyquist are ignored, as a C2R does.
      float2 xk = B[k * PR + r], xm = B[(hx - k) * PR + r];
      if (k == 0) { xk.y = 0.f; xm.y = 0.f; }
      xm.y = -xm.y;
      float2 e = cadd(xk, xm);
      float2 wk = __ldg(a.post + k);
      wk.y = -wk.y;
      float2 o = cmul(csub(xk, xm), wk);
      v = make_float2(e.x - o.y, e.y + o.x);
    } else {
      if (k == 0) v = make_float2(B[r].x, 0.f);
      else if (k < cnxp) v = B[k * PR + r];
      else { v = B[(hx - k) * PR + r]; v.y = -v.y; }
    }
    A[k * PR + r] = v;
  }
  __syncthreads();
  res = A;
  if (nr > 0) res = stockham<1, true>(A, 1, PR, B, 1, PR, a.rx, a.twx, nr) ? B : A;
  float *out = a.dst_r[gi] + (long long)z * nyp * a.rnxp;
  const float *add = a.add[gi] ? a.add[gi] + (long long)z * nyp * a.rnxp : nullptr;
  const float sc = a.scale[gi];
  const int ld = hx + 1;
  for (int idx = tid; idx < nr * ld; idx += nth) {
    const int r = (int)fdiv((uint32_t)idx, a.f_hx1), m = idx - r * ld;
    const long long ro = (long long)(y0 + r) * a.rnxp;
    if (a.even) {
      float2 v = make_float2(0.f, 0.f);
      if (m < hx) {
        v = cscale(res[m * PR + r], sc);
        if (add) v = cadd(v, reinterpret_cast<const float2 *>(add + ro)[m]);
      }
      reinterpret_cast<float2 *>(out + ro)[m] = v;
    } else {
      float v = 0.f;
      if (m < hx) {
        v = res[m * PR + r].x * sc;
        if (add) v += add[ro + m];
      }
      out[ro + m] = v;
    }
  }
  }  // items
}

// ------------------------------------------------------------------ z + solve
struct ZArgs {
  float2 *w[kMaxUnitGrids];
  int NP, nyp, nzp, zgroup;
  FastDiv f_nzp;
  RadixList rz;
  const float2 *twz;
  SolveConsts c;
  KzTables t;
  DevCounters *counters;
};

template <int DIR>
__device__ __forceinline__ void z_transform(float2 *D, float2 *Sx, int G, int ng_total, int zgroup,
                                            const RadixList &rz, const float2 *tw, int nzp) {
  for (int g0 = 0; g0 < ng_total; g0 += zgroup) {
    const int ng = min(zgroup, ng_total - g0);
    const int which = stockham<DIR, true>(D + 2 * g0, 1, 2 * G, Sx, 1, 2 * ng, rz, tw, 2 * ng);
    if (which) {
      for (int idx = threadIdx.x; idx < nzp * 2 * ng; idx += blockDim.x) {
        int zz = idx / (2 * ng), l = idx - zz * 2 * ng;
        D[zz * 2 * G + 2 * g0 + l] = Sx[idx];
      }
      __syncthreads();
    }
  }
}

template <int NT, int PREC>
__global__ void __launch_bounds__(kThreads) k_zsolve(const __grid_constant__ ZArgs a) {
  constexpr int G = 10 + NT;
  extern __shared__ float4 sm4[];
  const int nzp = a.nzp;
  float2 *D = reinterpret_cast<float2 *>(sm4);  // [z][G][2]
  float2 *Sx = D + (size_t)nzp * G * 2;         // [z][zgroup][2]
  float2 *tw = Sx + (size_t)nzp * a.zgroup * 2; // nzp
  const long long tile = blockIdx.x;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int idx = tid; idx < G * nzp; idx += nth) {
    const int g = (int)fdiv((uint32_t)idx, a.f_nzp), zz = idx - g * nzp;
    cp_async16(D + (zz * G + g) * 2, a.w[g] + (tile * nzp + zz) * 2);
  }
  for (int i = tid; i < nzp; i += nth) tw[i] = a.twz[i];
  cp_async_wait_all();
  __syncthreads();

  z_transform<-1>(D, Sx, G, G, a.zgroup, a.rz, tw, nzp);

  for (int b = tid; b < 2 * nzp; b += nth) {
    const int zz = b >> 1, t = b & 1;
    float2 *e = D + zz * 2 * G + t;  // grid g at e[2 g]
    float2 mu[3], d[NT], c6[6];
#pragma unroll
    for (int q = 0; q < 3; ++q) mu[q] = e[2 * q];
#pragma unroll
    for (int l = 0; l < NT; ++l) d[l] = e[2 * (3 + l)];
#pragma unroll
    for (int q = 0; q < 6; ++q) c6[q] = e[2 * (3 + NT + q)];
    const float2 ec = e[2 * (9 + NT)];
    const long long o = (long long)zz * NT;
    const bool fail = sb::solve_bin<NT, PREC>(a.c, a.t.wd + o, a.t.e1 + o, a.t.e2 + o, a.t.e3 + o,
                                              a.t.inv[zz] != 0, mu, d, c6, ec);
    bool nonfinite = false;
#pragma unroll
    for (int q = 0; q < 3; ++q) { e[2 * q] = mu[q]; nonfinite |= !sb::fin2(mu[q]); }
#pragma unroll
    for (int l = 0; l < NT; ++l) { e[2 * (3 + l)] = d[l]; nonfinite |= !sb::fin2(d[l]); }
#pragma unroll
    for (int q = 0; q < 6; ++q) { e[2 * (3 + NT + q)] = c6[q]; nonfinite |= !sb::fin2(c6[q]); }
    if (a.counters) sb::count(a.counters, fail, nonfinite);
  }
  __syncthreads();

  z_transform<1>(D, Sx, G, G - 1, a.zgroup, a.rz, tw, nzp);

  for (int idx = tid; idx < (G - 1) * nzp; idx += nth) {
    const int g = (int)fdiv((uint32_t)idx, a.f_nzp), zz = idx - g * nzp;
    const float4 v = *reinterpret_cast<const float4 *>(D + (zz * G + g) * 2);
    *reinterpret_cast<float4 *>(a.w[g] + (tile * nzp + zz) * 2) = v;
  }
}

template <typename Kern>
int launch_cluster(Kern kern, int nitems, int cs, size_t smem, cudaStream_t s, const PlaneArgs &a) {
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kPlaneThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // one cluster per (grid, z-plane) item
  cfg.gridDim = dim3(nitems * cs);
  CRAVA_CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, a));
  note_launch();
  return CRAVA_GPU_OK;
}

void fill_plane_args(const UnitPlan &p, const FftPlans &f, PlaneArgs *a) {
  const Geom &g = p.g;
  a->nxp = g.nxp; a->nyp = g.nyp; a->nzp = g.nzp; a->cnxp = g.cnxp; a->rnxp = g.rnxp;
  a->hx = p.hx; a->even = p.even; a->NP = p.NP; a->CS = p.CS; a->R = p.R; a->PP = p.PP;
  a->PR = p.PR; a->PC = p.PC; a->SA = p.SA; a->SB = p.SB; a->SC = p.SC;
  a->f_hx = make_fastdiv((uint32_t)p.hx);
  a->f_hx1 = make_fastdiv((uint32_t)(p.hx + 1));
  a->f_cnxp = make_fastdiv((uint32_t)g.cnxp);
  a->f_nyp = make_fastdiv((uint32_t)g.nyp);
  a->f_PP = make_fastdiv((uint32_t)p.PP);
  a->f_R = make_fastdiv((uint32_t)p.R);
  a->f_nzp = make_fastdiv((uint32_t)g.nzp);
  a->rx = f.x.rl; a->ry = f.y.rl;
  a->twx = f.x.tw; a->twy = f.y.tw; a->post = f.xpost;
}

}  // namespace

// Shared-memory need (float2) of the plane kernels for cluster size cs.
static void plane_sizes(const Geom &g, int hx, int NP, int cs, int *R, int *PP, int *PR, int *PC,
                        int *SA, int *SB, int *SC) {
  *R = (g.nyp + cs - 1) / cs;
  *PP = (NP + cs - 1) / cs;
  *PR = *R | 1;            // odd pitch
  *PC = 2 * *PP + 1;       // odd pitch
  *SA = std::max(hx * *PR, g.nyp * *PC);
  *SB = std::max(hx, g.cnxp) * *PR;
  *SC = g.nyp * *PC;
}

bool unit_plan(const Geom &g, int ntheta, UnitPlan *p) {
  p->g = g;
  p->even = (g.nxp % 2) == 0;
  p->hx = p->even ? g.nxp / 2 : g.nxp;
  p->NP = (g.cnxp + 1) / 2;
  p->ok = false;
  const size_t kMaxSmem = 227 * 1024;
  const size_t kTwoPerSm = 113 * 1024;
  int best = -1;
  for (int cs : {1, 2, 4, 8}) {
    if (cs > g.nyp) break;
    int R, PP, PR, PC, SA, SB, SC;
    plane_sizes(g, p->hx, p->NP, cs, &R, &PP, &PR, &PC, &SA, &SB, &SC);
    size_t smem = (size_t)(SA + SB + SC) * sizeof(float2);
    if (smem <= kTwoPerSm) { best = cs; break; }
    if (smem <= kMaxSmem && best < 0) best = cs;
  }
  if (best < 0) return false;
  p->CS = best;
  plane_sizes(g, p->hx, p->NP, best, &p->R, &p->PP, &p->PR, &p->PC, &p->SA, &p->SB, &p->SC);
  p->plane_smem = (size_t)(p->SA + p->SB + p->SC) * sizeof(float2);
  const int G = 10 + ntheta;
  const size_t data = (size_t)g.nzp * G * 2 * sizeof(float2) + (size_t)g.nzp * sizeof(float2);
  if (data + (size_t)g.nzp * 2 * sizeof(float2) > kMaxSmem) return false;
  int zg = (int)((kMaxSmem - data) / ((size_t)g.nzp * 2 * sizeof(float2)));
  zg = std::min(zg, G);
  p->zgroup = zg;
  p->z_smem = data + (size_t)g.nzp * zg * 2 * sizeof(float2);
  p->wgrid = (long long)g.nyp * p->NP * 2 * g.nzp;
  p->ok = true;
  return true;
}

int unit_plane_forward(const UnitPlan &p, const FftPlans &f, const float *const *src,
                       float2 *const *w, const float *scale, int n, cudaStream_t s) {
  if (n < 1 || n > kMaxUnitGrids) return CRAVA_GPU_ERR_ARG;
  PlaneArgs a{};
  fill_plane_args(p, f, &a);
  for (int i = 0; i < n; ++i) { a.src_r[i] = src[i]; a.w[i] = w[i]; a.scale[i] = scale[i]; }
  a.nitems = n * p.g.nzp;
  { int rc = func_smem((const void *)k_plane_fwd, p.plane_smem); if (rc) return rc; }
  return launch_cluster(k_plane_fwd, a.nitems, p.CS, p.plane_smem, s, a);
}

int unit_plane_inverse(const UnitPlan &p, const FftPlans &f, const float2 *const *w,
                       float *const *dst, const float *scale, const float *const *addend,
                       int n, cudaStream_t s) {
  if (n < 1 || n > kMaxUnitGrids) return CRAVA_GPU_ERR_ARG;
  PlaneArgs a{};
  fill_plane_args(p, f, &a);
  for (int i = 0; i < n; ++i) {
    a.w[i] = const_cast<float2 *>(w[i]);
    a.dst_r[i] = dst[i];
    a.scale[i] = scale[i];
    a.add[i] = addend ? addend[i] : nullptr;
  }
  a.nitems = n * p.g.nzp;
  { int rc = func_smem((const void *)k_plane_inv, p.plane_smem); if (rc) return rc; }
  return launch_cluster(k_plane_inv, a.nitems, p.CS, p.plane_smem, s, a);
}

template <int PREC>
static int launch_z(const ZArgs &a, int nt, const UnitPlan &p, cudaStream_t s) {
  const dim3 grd((unsigned)(p.NP * p.g.nyp));
  const int smem = (int)p.z_smem;
#define CRAVA_Z_CASE(N)                                                                       \
  case N:                                                                                     \
    { int rc_ = func_smem((const void *)k_zsolve<N, PREC>, (size_t)smem); if (rc_) return rc_; } \
    k_zsolve<N, PREC><<<grd, kThreads, smem, s>>>(a);                                         \
    break;
  switch (nt) {
    CRAVA_Z_CASE(1) CRAVA_Z_CASE(2) CRAVA_Z_CASE(3) CRAVA_Z_CASE(4)
    CRAVA_Z_CASE(5) CRAVA_Z_CASE(6) CRAVA_Z_CASE(7) CRAVA_Z_CASE(8)
    default: return CRAVA_GPU_ERR_ARG;
  }
#undef CRAVA_Z_CASE
  CRAVA_LAUNCH_CHECK();
  return CRAVA_GPU_OK;
}

int unit_zsolve(const UnitPlan &p, const FftPlans &f, const SolveConsts &c, const KzTables &t,
                float2 *const *w, int precision, DevCounters *counters, cudaStream_t s) {
  const int G = 10 + c.nt;
  ZArgs a{};
  for (int i = 0; i < G; ++i) a.w[i] = w[i];
  a.NP = p.NP; a.nyp = p.g.nyp; a.nzp = p.g.nzp; a.zgroup = p.zgroup;
  a.f_nzp = make_fastdiv((uint32_t)p.g.nzp);
  a.rz = f.z.rl; a.twz = f.z.tw;
  a.c = c; a.t = t; a.counters = counters;
  if (precision == CRAVA_SOLVE_FP64) return launch_z<0>(a, c.nt, p, s);
  if (precision == CRAVA_SOLVE_MIXED) return launch_z<1>(a, c.nt, p, s);
  return CRAVA_GPU_ERR_ARG;
}

}  // namespace crava
