// Group neighbour lists: the B200 counterpart of ORAC's linked-cell list
// (lc_index src/lc_index.f:3-125, lc_list src/lc_list.f:1-237) and of the
// all-pairs 'u' update (src/mts_forces.f:57-65 with src/force.f:258-286).
//
// ORAC bins group centres into ncx*ncy*ncz cells and, for every group n,
// scans a precomputed stencil of cells keeping partners l > n whose
// minimum-image centre distance is below rcut.  Here:
//   k_cell_assign   cell of every group (ORAC's floor/wrap formula, FP64)
//   k_scan          exclusive prefix sum (one block; lists are rebuilt every
//                   few steps, so one block is enough)
//   k_cell_fill     counting-sort placement, then k_cell_order sorts every
//                   cell by group index so results do not depend on atomics
//   k_pairs<FILL>   one warp per group, lanes over stencil cells; a count
//                   pass sizes the CSR rows, the fill pass writes them in
//                   stencil order and computes the exclusion masks of pairs
//                   that belong to one molecule.
// The stencil itself is built on the host with ORAC's dist_ijk criterion.
#include <algorithm>
#include <cmath>

#include "common.cuh"

namespace {

__device__ __forceinline__ int lc_cell(double x, double d, int nc) {
  // src/lc_list.f:94-102
  const double x1 = x / d;
  const int ix = (int)x1;
  const double frac = x1 - (double)ix;
  int n = ix + ((frac >= 0.0 ? 1 : -1) - 1) / 2;
  n %= nc;
  if (n < 0) n += nc;
  return n;
}

__global__ void k_cell_assign(int G, const double* __restrict__ grp, int ncx,
                              int ncy, int ncz, int* __restrict__ cell_of,
                              int* __restrict__ cell_cnt) {
  pdl_enter();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const int nx = lc_cell(grp[g], 2.0 / ncx, ncx);
  const int ny = lc_cell(grp[G + g], 2.0 / ncy, ncy);
  const int nz = lc_cell(grp[2 * G + g], 2.0 / ncz, ncz);
  const int c = nz + ncz * (ny + ncy * nx);
  cell_of[g] = c;
  atomicAdd(cell_cnt + c, 1);
}

// Exclusive scan of n ints into out[0..n], out[n] = total (also *total).
__global__ void __launch_bounds__(1024)
    k_scan(int n, const int* __restrict__ in, int* __restrict__ out,
           int64_t* __restrict__ total) {
  pdl_enter();
  __shared__ long long s[1024];
  const int t = threadIdx.x;
  const int chunk = (n + 1023) / 1024;
  const int b0 = t * chunk;
  const int b1 = min(n, b0 + chunk);
  long long sum = 0;
  for (int k = b0; k < b1; k++) sum += in[k];
  s[t] = sum;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    long long v = (t >= o) ? s[t - o] : 0;
    __syncthreads();
    s[t] += v;
    __syncthreads();
  }
  long long run = s[t] - sum;
  for (int k = b0; k < b1; k++) {
    const int v = in[k];
    out[k] = (int)run;
    run += v;
  }
  if (t == 1023) {
    out[n] = (int)s[1023];
    if (total) *total = s[1023];
  }
}

__global__ void k_cell_fill(int G, const int* __restrict__ cell_of,
                            const int* __restrict__ cell_start,
                            int* __restrict__ cursor, int* __restrict__ cell_grp) {
  pdl_enter();
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  const int c = cell_of[g];
  const int pos = cell_start[c] + atomicAdd(cursor + c, 1);
  cell_grp[pos] = g;
}

__global__ void k_cell_order(int ncell, const int* __restrict__ cell_start,
                             int* __restrict__ cell_grp) {
  pdl_enter();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int b = cell_start[c], e = cell_start[c + 1];
  for (int p = b + 1; p < e; p++) {  // insertion sort, cells hold few groups
    const int v = cell_grp[p];
    int q = p - 1;
    while (q >= b && cell_grp[q] > v) {
      cell_grp[q + 1] = cell_grp[q];
      q--;
    }
    cell_grp[q + 1] = v;
  }
}

struct ListArgs {
  int G;
  const double* grp;  // [3G] scaled
  double c11, c12, c13, c22, c23, c33;
  double rcut2;
  int ncx, ncy, ncz;
  const int* stencil;  // [3*nsten]
  int nsten;
  const int* cell_of;
  const int* cell_start;
  const int* cell_grp;
  // outputs
  int* cnt;
  const int* off;
  int* j;
  unsigned long long* mask;
  // topology for masks
  const int2* gmeta;
  const int* gmol;
  const int* exoff;
  const int* exj;
  const unsigned char* massinf;
  int allpairs;
  int64_t cap;  // fill pass: entries available (negative: unchecked)
  int* flag;    // fill pass: bit 1 set on overflow
};

__device__ __forceinline__ bool pair_in(const ListArgs& A, double xi, double yi,
                                        double zi, int l) {
  double dx = xi - A.grp[l], dy = yi - A.grp[A.G + l], dz = zi - A.grp[2 * A.G + l];
  dx -= 2.0 * round(0.5 * dx);  // pbc.h: anint(0.5 x)
  dy -= 2.0 * round(0.5 * dy);
  dz -= 2.0 * round(0.5 * dz);
  const double xx = A.c11 * dx + A.c12 * dy + A.c13 * dz;
  const double yy = A.c22 * dy + A.c23 * dz;
  const double zz = A.c33 * dz;
  return xx * xx + yy * yy + zz * zz < A.rcut2;
}

// Skip mask of pair (i, l) of one molecule: excluded atom pairs (mapnl), and
// for an i atom with any excluded partner in l, the pairs whose two masses
// are both >= massinfty (src/force.f:374-388, 486-489).
__device__ unsigned long long pair_mask(const ListArgs& A, int i, int l) {
  if (A.gmol[i] != A.gmol[l]) return 0ull;
  const int2 mi = A.gmeta[i], ml = A.gmeta[l];
  const int i0 = mi.x, ni = mi.y & 0xff, l0 = ml.x, nl = ml.y & 0xff;
  unsigned long long m = 0ull;
  for (int a = 0; a < ni; a++) {
    bool any = false;
    for (int e = A.exoff[i0 + a]; e < A.exoff[i0 + a + 1]; e++) {
      const int b = A.exj[e] - l0;
      if (b >= 0 && b < nl) {
        m |= 1ull << (a * 8 + b);
        any = true;
      }
    }
    if (any && A.massinf[i0 + a])
      for (int b = 0; b < nl; b++)
        if (A.massinf[l0 + b]) m |= 1ull << (a * 8 + b);
  }
  return m;
}

// One warp per group i.  Count pass: cnt[i].  Fill pass: entries in stencil
// order (lanes take 32 consecutive stencil cells, a warp scan orders their
// hits), within a cell by group index.
template <bool FILL>
__global__ void __launch_bounds__(128) k_pairs(const ListArgs A) {
  pdl_enter();
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (i >= A.G) return;
  if (FILL && A.cap >= 0 && (int64_t)A.off[A.G] > A.cap) {  // ORAC: xerror on nnlpp overflow
    if (i == 0 && lane == 0) atomicOr(A.flag, 2);
    return;
  }
  const double xi = A.grp[i], yi = A.grp[A.G + i], zi = A.grp[2 * A.G + i];
  int total = 0;
  const int base = FILL ? A.off[i] : 0;
  if (A.allpairs) {
    for (int l0 = i + 1; l0 < A.G; l0 += 32) {
      const int l = l0 + lane;
      const bool hit = l < A.G && pair_in(A, xi, yi, zi, l);
      const unsigned bal = __ballot_sync(0xffffffffu, hit);
      if (FILL && hit) {
        const int pos = base + total + __popc(bal & ((1u << lane) - 1u));
        A.j[pos] = l;
        A.mask[pos] = pair_mask(A, i, l);
      }
      total += __popc(bal);
    }
  } else {
    const int c = A.cell_of[i];
    const int ci = c / (A.ncy * A.ncz), cj = (c / A.ncz) % A.ncy, ck = c % A.ncz;
    for (int s0 = 0; s0 < A.nsten; s0 += 32) {
      const int s = s0 + lane;
      int cb = 0, ce = 0;
      if (s < A.nsten) {
        int nx = (ci + A.stencil[3 * s]) % A.ncx;
        if (nx < 0) nx += A.ncx;
        int ny = (cj + A.stencil[3 * s + 1]) % A.ncy;
        if (ny < 0) ny += A.ncy;
        int nz = (ck + A.stencil[3 * s + 2]) % A.ncz;
        if (nz < 0) nz += A.ncz;
        const int cc = nz + A.ncz * (ny + A.ncy * nx);
        cb = A.cell_start[cc];
        ce = A.cell_start[cc + 1];
      }
      int mine = 0;
      for (int p = cb; p < ce; p++) {
        const int l = A.cell_grp[p];
        if (l > i && pair_in(A, xi, yi, zi, l)) mine++;
      }
      // exclusive warp scan of the per-lane hit counts
      int incl = mine;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      if (FILL && mine) {
        int pos = base + total + incl - mine;
        for (int p = cb; p < ce; p++) {
          const int l = A.cell_grp[p];
          if (l > i && pair_in(A, xi, yi, zi, l)) {
            A.j[pos] = l;
            A.mask[pos] = pair_mask(A, i, l);
            pos++;
          }
        }
      }
      total += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
  if (!FILL && lane == 0) A.cnt[i] = total;
}

// dist_ijk (src/dist_ijk.f:3-141): squared minimum distance between cell
// (0,0,0) and cell (ni,nj,nk) from corner pairs, refined along the edges.
double dist_ijk(int ni, int nj, int nk, double dx, double dy, double dz, const double* co) {
  static const int nv[8][3] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                               {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
  const int ndtmax = 500;
  double dmin = 1e8;
  int imin = 0, jmin = 0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const double lx = (ni + nv[j][0] - nv[i][0]) * dx;
      const double ly = (nj + nv[j][1] - nv[i][1]) * dy;
      const double lz = (nk + nv[j][2] - nv[i][2]) * dz;
      const double mx = co[0] * lx + co[3] * ly + co[6] * lz;
      const double my = co[1] * lx + co[4] * ly + co[7] * lz;
      const double mz = co[2] * lx + co[5] * ly + co[8] * lz;
      const double d = mx * mx + my * my + mz * mz;
      if (d < dmin) {
        dmin = d;
        imin = i;
        jmin = j;
      }
    }
  const double lx = (ni + nv[jmin][0] - nv[imin][0]) * dx;
  const double ly = (nj + nv[jmin][1] - nv[imin][1]) * dy;
  const double lz = (nk + nv[jmin][2] - nv[imin][2]) * dz;
  const double mx = co[0] * lx + co[3] * ly + co[6] * lz;
  const double my = co[1] * lx + co[4] * ly + co[7] * lz;
  const double mz = co[2] * lx + co[5] * ly + co[8] * lz;
  dmin = 1e8;
  const double steps[3] = {dx, dy, dz};
  for (int ax = 0; ax < 3; ax++) {
    const double dt = ((0.5 - nv[jmin][ax]) >= 0 ? 1.0 : -1.0) * steps[ax] / ndtmax;
    for (int i = 1; i <= ndtmax; i++) {
      const double dmx = i * co[0 + 3 * ax] * dt;
      const double dmy = i * co[1 + 3 * ax] * dt;
      const double dmz = i * co[2 + 3 * ax] * dt;
      const double d = (mx + dmx) * (mx + dmx) + (my + dmy) * (my + dmy) + (mz + dmz) * (mz + dmz);
      if (d < dmin) dmin = d;
    }
  }
  return dmin;
}

// Full stencil of lc_index (src/lc_index.f:52-91, n = 2) with its
// double-visit check (src/lc_index.f:106-122).
int build_stencil(orac_gpu_ctx* ctx, double rcut) {
  const int ncx = ctx->ncx, ncy = ctx->ncy, ncz = ctx->ncz;
  if (ctx->d_stencil && ctx->sten_rcut == rcut && ctx->sten_nc[0] == ncx && ctx->sten_nc[1] == ncy &&
      ctx->sten_nc[2] == ncz && memcmp(ctx->sten_co, ctx->co, sizeof(ctx->co)) == 0)
    return ORAC_OK;
  const double sq = rcut * rcut, dx = 2.0 / ncx, dy = 2.0 / ncy, dz = 2.0 / ncz;
  std::vector<int> st = {0, 0, 0};
  int imax = 0, jmax = 0, kmax = 0;
  for (int i = 1 - ncx; i <= ncx - 1; i++)
    for (int j = 1 - ncy; j <= ncy - 1; j++)
      for (int k = 1 - ncz; k <= ncz - 1; k++) {
        if (dist_ijk(i, j, k, dx, dy, dz, ctx->co) < sq) {
          if (i == 0 && j == 0 && k == 0) continue;
          st.push_back(i);
          st.push_back(j);
          st.push_back(k);
          imax = std::max(imax, std::abs(i));
          jmax = std::max(jmax, std::abs(j));
          kmax = std::max(kmax, std::abs(k));
        }
      }
  if (imax >= (ncx + 1) / 2 || jmax >= (ncy + 1) / 2 || kmax >= (ncz + 1) / 2)
    return ctx_fail(ctx, ORAC_ERR_PARAM,
                    "linked cells %dx%dx%d too coarse for rcut %.3f: a cell would be visited twice "
                    "(ORAC lc_index stops here)",
                    ncx, ncy, ncz, rcut);
  if (dev_alloc(ctx, &ctx->d_stencil, st.size())) return ORAC_ERR_CUDA;
  CK(cudaMemcpyAsync(ctx->d_stencil, st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  ctx->nsten = (int)st.size() / 3;
  ctx->sten_rcut = rcut;
  ctx->sten_nc[0] = ncx;
  ctx->sten_nc[1] = ncy;
  ctx->sten_nc[2] = ncz;
  memcpy(ctx->sten_co, ctx->co, sizeof(ctx->co));
  return ORAC_OK;
}

ListArgs base_args(orac_gpu_ctx* ctx, double rcut, GList* out) {
  ListArgs A;
  memset(&A, 0, sizeof(A));
  A.G = ctx->G;
  A.grp = ctx->d_grp;
  A.c11 = ctx->co[0];
  A.c12 = ctx->co[3];
  A.c13 = ctx->co[6];
  A.c22 = ctx->co[4];
  A.c23 = ctx->co[7];
  A.c33 = ctx->co[8];
  A.rcut2 = rcut * rcut;
  A.ncx = ctx->ncx;
  A.ncy = ctx->ncy;
  A.ncz = ctx->ncz;
  A.stencil = ctx->d_stencil;
  A.nsten = ctx->nsten;
  A.cell_of = ctx->d_cell_of;
  A.cell_start = ctx->d_cell_start;
  A.cell_grp = ctx->d_cell_grp;
  A.cnt = out->cnt;
  A.off = out->off;
  A.gmeta = ctx->d_gmeta;
  A.gmol = ctx->d_gmol;
  A.exoff = ctx->d_exoff;
  A.exj = ctx->d_exj;
  A.massinf = ctx->d_amassinf;
  A.cap = -1;
  A.flag = ctx->d_flag;
  return A;
}

// count -> scan -> (grow) -> fill
int pairs_count_fill(orac_gpu_ctx* ctx, ListArgs A, GList* out) {
  const int nb = (ctx->G + 3) / 4;
  orac_launch(k_pairs<false>, nb, 128, 0, ctx->stream, A);
  CKL();
  orac_launch(k_scan, 1, 1024, 0, ctx->stream, ctx->G, out->cnt, out->off, ctx->d_total);
  CKL();
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, ctx->d_total, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (total >= (int64_t)1 << 31) return ctx_fail(ctx, ORAC_ERR_CAPACITY, "neighbour list of %lld pairs", (long long)total);
  if (total > out->cap) {
    const int64_t cap = total + total / 4 + 1024;
    if (dev_alloc(ctx, &out->j, cap)) return ORAC_ERR_CUDA;
    if (dev_alloc(ctx, &out->mask, cap)) return ORAC_ERR_CUDA;
    out->cap = cap;
    // nested lists share the rows of this list and need the same capacity
    for (int q = 1; q < 3; q++) {
      GList& L = ctx->lists[q];
      if (dev_alloc(ctx, &L.j, cap)) return ORAC_ERR_CUDA;
      if (dev_alloc(ctx, &L.mask, cap)) return ORAC_ERR_CUDA;
      L.cap = cap;
      L.valid = false;
    }
  }
  A.j = out->j;
  A.mask = out->mask;
  orac_launch(k_pairs<true>, nb, 128, 0, ctx->stream, A);
  CKL();
  out->npairs = total;
  out->valid = true;
  ctx->lists[1].valid = false;
  ctx->lists[2].valid = false;
  return ORAC_OK;
}

}  // namespace

int list_build_cells(orac_gpu_ctx* ctx, double rcut, GList* out) {
  if (int rc = build_stencil(ctx, rcut)) return rc;
  const int ncell = ctx->ncx * ctx->ncy * ctx->ncz;
  if (ncell > ctx->ncell_cap) {
    if (dev_alloc(ctx, &ctx->d_cell_cnt, ncell + 1)) return ORAC_ERR_CUDA;
    if (dev_alloc(ctx, &ctx->d_cell_start, ncell + 1)) return ORAC_ERR_CUDA;
    ctx->ncell_cap = ncell;
  }
  CK(cudaMemsetAsync(ctx->d_cell_cnt, 0, sizeof(int) * (ncell + 1), ctx->stream));
  const int G = ctx->G;
  orac_launch(k_cell_assign, (G + 255) / 256, 256, 0, ctx->stream, G, ctx->d_grp, ctx->ncx, ctx->ncy, ctx->ncz,
                                                         ctx->d_cell_of, ctx->d_cell_cnt);
  CKL();
  orac_launch(k_scan, 1, 1024, 0, ctx->stream, ncell, ctx->d_cell_cnt, ctx->d_cell_start, nullptr);
  CKL();
  CK(cudaMemsetAsync(ctx->d_cell_cnt, 0, sizeof(int) * (ncell + 1), ctx->stream));
  orac_launch(k_cell_fill, (G + 255) / 256, 256, 0, ctx->stream, G, ctx->d_cell_of, ctx->d_cell_start, ctx->d_cell_cnt,
                                                       ctx->d_cell_grp);
  CKL();
  orac_launch(k_cell_order, (ncell + 255) / 256, 256, 0, ctx->stream, ncell, ctx->d_cell_start, ctx->d_cell_grp);
  CKL();
  ListArgs A = base_args(ctx, rcut, out);
  A.allpairs = 0;
  return pairs_count_fill(ctx, A, out);
}

int list_build_allpairs(orac_gpu_ctx* ctx, double rcut, GList* out) {
  ListArgs A = base_args(ctx, rcut, out);
  A.allpairs = 1;
  return pairs_count_fill(ctx, A, out);
}

int list_prepare_stencil(orac_gpu_ctx* ctx, double rcut) {
  if (int rc = build_stencil(ctx, rcut)) return rc;
  const int ncell = ctx->ncx * ctx->ncy * ctx->ncz;
  if (ncell > ctx->ncell_cap) {
    if (dev_alloc(ctx, &ctx->d_cell_cnt, ncell + 1)) return ORAC_ERR_CUDA;
    if (dev_alloc(ctx, &ctx->d_cell_start, ncell + 1)) return ORAC_ERR_CUDA;
    ctx->ncell_cap = ncell;
  }
  return ORAC_OK;
}

int list_build_cells_async(orac_gpu_ctx* ctx, double rcut, GList* out, int* d_flag) {
  if (!ctx->d_stencil || ctx->sten_rcut != rcut)
    return ctx_fail(ctx, ORAC_ERR_STATE, "stencil for rcut %.3f not prepared", rcut);
  const int ncell = ctx->ncx * ctx->ncy * ctx->ncz;
  const int G = ctx->G;
  CK(cudaMemsetAsync(ctx->d_cell_cnt, 0, sizeof(int) * (ncell + 1), ctx->stream));
  orac_launch(k_cell_assign, (G + 255) / 256, 256, 0, ctx->stream, G, ctx->d_grp, ctx->ncx, ctx->ncy, ctx->ncz,
                                                         ctx->d_cell_of, ctx->d_cell_cnt);
  CKL();
  orac_launch(k_scan, 1, 1024, 0, ctx->stream, ncell, ctx->d_cell_cnt, ctx->d_cell_start, nullptr);
  CKL();
  CK(cudaMemsetAsync(ctx->d_cell_cnt, 0, sizeof(int) * (ncell + 1), ctx->stream));
  orac_launch(k_cell_fill, (G + 255) / 256, 256, 0, ctx->stream, G, ctx->d_cell_of, ctx->d_cell_start, ctx->d_cell_cnt,
                                                       ctx->d_cell_grp);
  CKL();
  orac_launch(k_cell_order, (ncell + 255) / 256, 256, 0, ctx->stream, ncell, ctx->d_cell_start, ctx->d_cell_grp);
  CKL();
  ListArgs A = base_args(ctx, rcut, out);
  A.allpairs = 0;
  A.cap = out->cap;
  A.flag = d_flag;
  const int nb = (G + 3) / 4;
  orac_launch(k_pairs<false>, nb, 128, 0, ctx->stream, A);
  CKL();
  orac_launch(k_scan, 1, 1024, 0, ctx->stream, G, out->cnt, out->off, ctx->d_total);
  CKL();
  A.j = out->j;
  A.mask = out->mask;
  orac_launch(k_pairs<true>, nb, 128, 0, ctx->stream, A);
  CKL();
  out->valid = true;
  return ORAC_OK;
}
