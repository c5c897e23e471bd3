// Smooth particle-mesh Ewald on the GPU: the counterpart of ORAC's FFTW
// build of do_pmesh_kspace (src/pme_fftw3.f90:56-130) with scalar_sum
// (src/scalar_sum.f:2-135), replacing FFTW by a shared-memory FFT.
//
//   k_spread      fractional coordinates in FP64 (get_scaled_fractionals,
//                 pme_fftw3.f90:132-163), cardinal B-splines in FP32
//                 (fill_bspline :518-576), charge spreading with 64-bit
//                 fixed-point atomics (fill_charge_grid :233-298) so the grid
//                 does not depend on the order of the atomics
//   k_fft<MODE>   Stockham mixed-radix (2,3,4,5,7) FFT of batches of grid lines
//                 held in shared memory; MODE selects the axis and the
//                 r2c / c2c / c2r form.  FFTW's conventions: r2c forward
//                 exp(-i..) along the fastest axis n1 giving (n1/2+1,n2,n3),
//                 c2r backward, unnormalised.
//   ZCONV         the z pass runs forward FFT, the influence function of
//                 scalar_sum (energy and virial with ORAC's fac12/13/23
//                 masks, FP64 reductions) and the inverse FFT on the same
//                 lines without leaving shared memory
//   k_gather      forces (grad_sum :310-372) and the molecular virial
//                 correction of fft_pme (src/fft_pme.f:65-106)
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int MAXR = 12;  // max radix stages
constexpr int FFT_THREADS = 128;

// Division by a constant of the plan: q = umulhi(t, m) with m = 2^32/d + 1
// is floor(t / d) whenever t * d < 2^32 (here t < 2^20, d <= 4096).  That m
// does not fit 32 bits for d = 1, which is marked by m = 0.
inline unsigned magic_of(unsigned d) { return d == 1 ? 0u : (unsigned)((1ull << 32) / d + 1ull); }
__device__ __forceinline__ int qdiv(int t, unsigned m) { return m ? (int)__umulhi((unsigned)t, m) : t; }

struct FftPlan {
  int n;
  int nst;
  int rad[MAXR];
  // per stage: butterflies per line, span of the finished sub-transforms,
  // twiddle stride, and the division constants of the first two
  int nb[MAXR], ns[MAXR], tsc[MAXR];
  unsigned mnb[MAXR], mns[MAXR];
  unsigned mn;  // division by n
};

int make_plan(int n, FftPlan* p) {
  p->n = n;
  p->nst = 0;
  int m = n;
  while (m % 4 == 0 && p->nst < MAXR) {
    p->rad[p->nst++] = 4;
    m /= 4;
  }
  const int rs[] = {2, 3, 5, 7};
  for (int r : rs)
    while (m % r == 0 && p->nst < MAXR) {
      p->rad[p->nst++] = r;
      m /= r;
    }
  if (m != 1 || n > 2048) return -1;  // 3 lines of 2048 complex values fill 48 KB of shared memory
  int ns = 1;
  for (int s = 0; s < p->nst; s++) {
    const int R = p->rad[s];
    p->nb[s] = n / R;
    p->ns[s] = ns;
    p->tsc[s] = n / (ns * R);
    p->mnb[s] = magic_of((unsigned)p->nb[s]);
    p->mns[s] = magic_of((unsigned)ns);
    ns *= R;
  }
  p->mn = magic_of((unsigned)n);
  return 0;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// W_n^k for sign -1 (forward) is tw[k] (0 <= k < n); sign +1 takes the
// conjugate.
__device__ __forceinline__ float2 twid(const float2* tw, int k, int sign) {
  float2 w = tw[k];
  if (sign > 0) w.y = -w.y;
  return w;
}

// One Stockham pass of radix R over nl lines of length n (line-major, a ->
// b): butterfly t = (line l, index j < n/R) reads a[l][j + r n/R], applies
// the twiddles W_n^(k r tsc) with k = j mod Ns, and writes the R-point DFT
// to b[l][(j/Ns) Ns R + k + q Ns].
template <int R>
__device__ __forceinline__ void fft_pass(const float2* __restrict__ in, float2* __restrict__ out, int nl, int n,
                                         const FftPlan& P, int s, const float2* tw, int sign) {
  const int nb = P.nb[s], Ns = P.ns[s], tsc = P.tsc[s];
  const unsigned mnb = P.mnb[s], mns = P.mns[s];
  float2 wr[R];  // W_R^m = W_n^(m nb)
#pragma unroll
  for (int m = 0; m < R; m++) wr[m] = twid(tw, m * nb, sign);
  const int tot = nl * nb;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int l = qdiv(t, mnb), j = t - l * nb;
    const int jq = qdiv(j, mns), k = j - jq * Ns;
    const int tstep = k * tsc;
    const float2* src = in + l * n + j;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      float2 x = src[r * nb];
      if (r && tstep) x = cmul(x, twid(tw, tstep * r, sign));
      v[r] = x;
    }
    float2* dst = out + l * n + jq * Ns * R + k;
    if (R == 2) {
      dst[0] = cadd(v[0], v[1]);
      dst[Ns] = csub(v[0], v[1]);
    } else if (R == 4) {
      const float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
      const float2 s13 = cadd(v[1], v[3]), d13 = csub(v[1], v[3]);
      // -i*sign(-1) d13 : forward multiplies by -i, inverse by +i
      const float2 rot = sign < 0 ? make_float2(d13.y, -d13.x) : make_float2(-d13.y, d13.x);
      dst[0] = cadd(s02, s13);
      dst[Ns] = cadd(d02, rot);
      dst[2 * Ns] = csub(s02, s13);
      dst[3 * Ns] = csub(d02, rot);
    } else {
#pragma unroll
      for (int q = 0; q < R; q++) {
        float2 acc = v[0];
#pragma unroll
        for (int r = 1; r < R; r++) acc = cadd(acc, cmul(v[r], wr[(r * q) % R]));
        dst[q * Ns] = acc;
      }
    }
  }
}

// Stockham passes over `nl` lines of length n stored line-major in a; the
// result ends in the returned buffer (a or b).
__device__ float2* fft_smem(float2* a, float2* b, int nl, const FftPlan& P, const float2* tw, int sign) {
  const int n = P.n;
  for (int s = 0; s < P.nst; s++) {
    switch (P.rad[s]) {
      case 4: fft_pass<4>(a, b, nl, n, P, s, tw, sign); break;
      case 2: fft_pass<2>(a, b, nl, n, P, s, tw, sign); break;
      case 3: fft_pass<3>(a, b, nl, n, P, s, tw, sign); break;
      case 5: fft_pass<5>(a, b, nl, n, P, s, tw, sign); break;
      default: fft_pass<7>(a, b, nl, n, P, s, tw, sign); break;
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

__device__ __forceinline__ double warp_sumd(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block reduction of NV doubles into out[] with atomics.
template <int NV>
__device__ void block_reduce_add(double* v, double* out) {
  __shared__ double s[32][NV];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) {
    const double x = warp_sumd(v[q]);
    if (lane == 0) s[w][q] = x;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double x = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) x += s[k][threadIdx.x];
    if (x != 0.0) atomicAdd(out + threadIdx.x, x);
  }
}

struct GridArgs {
  int n1, n2, n3, h1;
  const unsigned long long* qfix;
  float2* cg;
  float* rg;
  const float2* tw;
  FftPlan P;
  int B;  // lines per block
  // convolution
  const float* bsp1;
  const float* bsp2;
  const float* bsp3;
  double r11, r12, r13, r21, r22, r23, r31, r32, r33;  // recip(i,j)
  float fac, pivol;  // pi^2/alpha^2, pi*volume
  double rkcut2;
  double* eout;  // [7] energy, v11 v22 v33 v12 v13 v23
  // the z pass keeps the transformed grid (save), or, given the transformed
  // grid S of other charges (cross), sums the energy difference
  // |S|^2 - |S - T|^2 = 2 Re(S conj T) - |T|^2 of this grid T and stops
  float2* save;
  const float2* cross;
};

enum { XF = 0, YF = 1, ZC = 2, YI = 3, XI = 4 };

template <int MODE>
__global__ void __launch_bounds__(FFT_THREADS) k_fft(const GridArgs A) {
  pdl_enter();
  extern __shared__ float2 sm[];
  const int n = A.P.n;
  const int B = A.B;
  float2* a = sm;
  float2* b = sm + B * n;
  // the line's twiddles, staged after the two line buffers
  float2* tws = sm + 2 * B * n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) tws[e] = A.tw[e];
  // line geometry
  int nlines, i0 = 0, j0 = 0, k0 = 0, nl;
  if (MODE == XF || MODE == XI) {
    nlines = A.n2 * A.n3;
    const int L0 = blockIdx.x * B;
    nl = min(B, nlines - L0);
    j0 = L0;  // linear (j + n2 k) of first line
  } else if (MODE == YF || MODE == YI) {
    const int nib = (A.h1 + B - 1) / B;
    k0 = blockIdx.x / nib;
    i0 = (blockIdx.x % nib) * B;
    nl = min(B, A.h1 - i0);
  } else {
    const int nib = (A.h1 + B - 1) / B;
    j0 = blockIdx.x / nib;
    i0 = (blockIdx.x % nib) * B;
    nl = min(B, A.h1 - i0);
  }
  const unsigned mnl = nl == 1 ? 0u : (unsigned)((1ull << 32) / (unsigned)nl + 1ull);  // division by nl
  // ---- load
  if (MODE == XF) {
    const size_t g0 = (size_t)j0 * A.n1;
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const long long q = (long long)A.qfix[g0 + e];
      a[e] = make_float2((float)((double)q * (1.0 / ORAC_QSCALE)), 0.f);
    }
  } else if (MODE == XI) {
    // Hermitian extension of the half line (c2r)
    const int h1 = A.h1;
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int l = qdiv(e, A.P.mn), i = e - l * n;
      const size_t row = (size_t)(j0 + l) * h1;
      float2 v;
      if (i < h1) {
        v = A.cg[row + i];
      } else {
        v = A.cg[row + (n - i)];
        v.y = -v.y;
      }
      a[e] = v;
    }
  } else if (MODE == YF || MODE == YI) {
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int pos = qdiv(e, mnl), l = e - pos * nl;
      a[l * n + pos] = A.cg[((size_t)k0 * A.n2 + pos) * A.h1 + i0 + l];
    }
  } else {
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int pos = qdiv(e, mnl), l = e - pos * nl;
      a[l * n + pos] = A.cg[((size_t)pos * A.n2 + j0) * A.h1 + i0 + l];
    }
  }
  __syncthreads();
  const int sign = (MODE == XF || MODE == YF) ? -1 : +1;
  float2* res = fft_smem(a, b, nl, A.P, tws, MODE == ZC ? -1 : sign);
  if (MODE == ZC) {
    // influence function, src/scalar_sum.f:40-121 (element (1,1,1) untouched)
    double acc[7] = {0, 0, 0, 0, 0, 0, 0};
    const int ndim1 = A.h1;
    int nf1 = A.n1 / 2;
    if (2 * nf1 < A.n1) nf1++;
    int nf2 = A.n2 / 2;
    if (2 * nf2 < A.n2) nf2++;
    int nf3 = A.n3 / 2;
    if (2 * nf3 < A.n3) nf3++;
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int l = qdiv(e, A.P.mn), kk = e - l * n;
      const int k1 = i0 + l + 1, k2 = j0 + 1, k3 = kk + 1;
      if (k1 == 1 && k2 == 1 && k3 == 1) continue;
      const int m1 = k1 > nf1 ? k1 - 1 - A.n1 : k1 - 1;
      const int m2 = k2 > nf2 ? k2 - 1 - A.n2 : k2 - 1;
      const int m3 = k3 > nf3 ? k3 - 1 - A.n3 : k3 - 1;
      const double mh1 = A.r11 * m1 + A.r12 * m2 + A.r13 * m3;
      const double mh2 = A.r21 * m1 + A.r22 * m2 + A.r23 * m3;
      const double mh3 = A.r31 * m1 + A.r32 * m2 + A.r33 * m3;
      const double msq = mh1 * mh1 + mh2 * mh2 + mh3 * mh3;
      float2 q = res[e];
      const size_t gi = ((size_t)kk * A.n2 + j0) * A.h1 + i0 + l;  // the element's place in cg
      if (A.save) A.save[gi] = q;
      float eterm = 0.f;
      if (msq <= A.rkcut2) {
        const float fm = (float)msq;
        const float denom = A.pivol * A.bsp1[k1 - 1] * A.bsp2[k2 - 1] * A.bsp3[k3 - 1] * fm;
        eterm = expf(-A.fac * fm) / denom;
        const double vterm = 2.0 * ((double)A.fac * msq + 1.0) / msq;
        double q2 = (double)q.x * q.x + (double)q.y * q.y;
        if (A.cross) {
          const float2 c = A.cross[gi];
          q2 = 2.0 * ((double)q.x * c.x + (double)q.y * c.y) - q2;
        }
        double struc2;
        double f12 = 1, f13 = 1, f23 = 1;
        if (k1 == 1 || (k1 == ndim1 && (A.n1 % 2) == 0)) {
          struc2 = (double)eterm * q2;
        } else {
          struc2 = 2.0 * (double)eterm * q2;
          f12 = (mh1 * mh2 < 0.0 && k2 <= ndim1) ? 0.0 : 1.0;
          f13 = (mh1 * mh3 < 0.0 && k3 <= ndim1) ? 0.0 : 1.0;
          const bool neg = mh2 * mh3 < 0.0;
          if (k2 <= ndim1 && k3 <= ndim1)
            f23 = neg ? 0.0 : 1.0;
          else if (k2 > ndim1 && k3 <= ndim1)
            f23 = neg ? 1.0 : 0.0;
          else if (k3 > ndim1 && k2 <= ndim1)
            f23 = neg ? 1.0 : 0.0;
          else
            f23 = neg ? 0.0 : 1.0;
        }
        const double vvir = struc2 * vterm;
        acc[0] += struc2;
        acc[1] += struc2 * (vterm * mh1 * mh1 - 1.0);
        acc[2] += struc2 * (vterm * mh2 * mh2 - 1.0);
        acc[3] += struc2 * (vterm * mh3 * mh3 - 1.0);
        acc[4] += vvir * mh1 * mh2 * f12;
        acc[5] += vvir * mh1 * mh3 * f13;
        acc[6] += vvir * mh2 * mh3 * f23;
      }
      res[e] = make_float2(q.x * eterm, q.y * eterm);
    }
    __syncthreads();
    block_reduce_add<7>(acc, A.eout);
    if (A.cross) return;  // the energy difference alone
    float2* other = (res == a) ? b : a;
    res = fft_smem(res, other, nl, A.P, tws, +1);
  }
  // ---- store
  if (MODE == XF) {
    const int h1 = A.h1;
    for (int e = threadIdx.x; e < nl * h1; e += blockDim.x) {
      const int l = e / h1, i = e - l * h1;
      A.cg[(size_t)(j0 + l) * h1 + i] = res[l * n + i];
    }
  } else if (MODE == XI) {
    const size_t g0 = (size_t)j0 * A.n1;
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) A.rg[g0 + e] = res[e].x;
  } else if (MODE == YF || MODE == YI) {
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int pos = qdiv(e, mnl), l = e - pos * nl;
      A.cg[((size_t)k0 * A.n2 + pos) * A.h1 + i0 + l] = res[l * n + pos];
    }
  } else {
    for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
      const int pos = qdiv(e, mnl), l = e - pos * nl;
      A.cg[((size_t)pos * A.n2 + j0) * A.h1 + i0 + l] = res[l * n + pos];
    }
  }
}

struct AtomArgs {
  int natom, order, n1, n2, n3;
  const double* xyz;  // [3N] Cartesian
  const double* q;
  double r11, r12, r13, r21, r22, r23, r31, r32, r33;
  unsigned long long* qfix;
  const float* rg;
  double* f;  // [3N] accumulated
  unsigned long long* ffix;  // [3N] fixed-point alternative to f (or null)
  // molecular correction (optional)
  const double* sxyz;  // [3N] scaled
  const double* mol;   // [3P] scaled
  const int* amol;
  int P;
  double c11, c12, c13, c22, c23, c33;
  double* eout;  // [7+9]
  // dE/dlambda of alchemical charges: sum_i phi_i dq_i/dlambda, with phi_i the
  // reciprocal potential at atom i (dE/dq_i), into *edq (both null: off)
  const double* dq;
  double* edq;
};

// fill_bspline restated in FP32 (src/pme_fftw3.f90:518-576).  P > 0: the
// order fixed at compile time (every loop unrolled, the arrays in
// registers); P = 0: the run-time order.  Both do the same operations.
constexpr int MAXORD = 12;

template <int P>
__device__ __forceinline__ void bspline(float w, int order_rt, float* c, float* d) {
  const int order = P > 0 ? P : order_rt;
  c[order - 1] = 0.f;
  c[1] = w;
  c[0] = 1.f - w;
#pragma unroll
  for (int k = 3; k <= (P > 0 ? P : MAXORD) - 1; k++) {
    if (P == 0 && k > order - 1) break;
    const float div = 1.f / (k - 1);
    c[k - 1] = div * w * c[k - 2];
#pragma unroll
    for (int j = 1; j <= k - 2; j++) c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
    c[0] = div * (1.f - w) * c[0];
  }
  d[0] = -c[0];
#pragma unroll
  for (int j = 2; j <= (P > 0 ? P : MAXORD); j++) {
    if (P == 0 && j > order) break;
    d[j - 1] = c[j - 2] - c[j - 1];
  }
  {
    const int k = order;
    const float div = 1.f / (k - 1);
    c[k - 1] = div * w * c[k - 2];
#pragma unroll
    for (int j = 1; j <= (P > 0 ? P : MAXORD) - 2; j++) {
      if (P == 0 && j > k - 2) break;
      c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
    }
    c[0] = div * (1.f - w) * c[0];
  }
}


__device__ __forceinline__ void frac_coord(const AtomArgs& A, int t, double* fr) {
  const double x = A.xyz[t], y = A.xyz[A.natom + t], z = A.xyz[2 * A.natom + t];
  double w = x * A.r11 + y * A.r21 + z * A.r31;
  fr[0] = A.n1 * (w - round(w) + 0.5);
  w = x * A.r12 + y * A.r22 + z * A.r32;
  fr[1] = A.n2 * (w - round(w) + 0.5);
  w = x * A.r13 + y * A.r23 + z * A.r33;
  fr[2] = A.n3 * (w - round(w) + 0.5);
}

// w - anint(w) + 0.5 lies in [0, 1] for finite w, so fr lies in [0, n]
__device__ __forceinline__ bool frac_ok(const AtomArgs& A, const double* fr) {
  return fr[0] >= 0.0 && fr[0] <= A.n1 && fr[1] >= 0.0 && fr[1] <= A.n2 && fr[2] >= 0.0 && fr[2] <= A.n3;
}

__device__ __forceinline__ int gidx(int k0, int n) {
  int k = k0 >= 0 ? k0 : k0 + n;
  if (k >= n) k -= n;  // fractional coordinate exactly at n
  return k;
}

// one thread per (atom, i3 plane); P > 0: the order at compile time (the
// spline arrays in registers), 0: A.order
template <int P>
__global__ void k_spread(const AtomArgs A) {
  pdl_enter();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int p = P > 0 ? P : A.order;
  if (t >= A.natom * p) return;
  const int at = t / p, i3 = t - at * p;
  double fr[3];
  frac_coord(A, at, fr);
  if (!frac_ok(A, fr)) return;  // non-finite coordinates never index the grid
  float th1[MAXORD], th2[MAXORD], th3[MAXORD], d[MAXORD];
  bspline<P>((float)(fr[0] - (int)fr[0]), p, th1, d);
  bspline<P>((float)(fr[1] - (int)fr[1]), p, th2, d);
  bspline<P>((float)(fr[2] - (int)fr[2]), p, th3, d);
  float t3 = 0.f;  // th3[i3], selected without a run-time index
#pragma unroll
  for (int k = 0; k < (P > 0 ? P : MAXORD); k++)
    if (k == i3) t3 = th3[k];
  const float qa = (float)A.q[at];
  const int kk = gidx((int)fr[2] - p + 1 + i3, A.n3);
#pragma unroll
  for (int i2 = 0; i2 < (P > 0 ? P : MAXORD); i2++) {
    if (P == 0 && i2 >= p) break;
    const int jj = gidx((int)fr[1] - p + 1 + i2, A.n2);
    const float prod = th2[i2] * t3 * qa;
    unsigned long long* row = A.qfix + ((size_t)kk * A.n2 + jj) * A.n1;
#pragma unroll
    for (int i1 = 0; i1 < (P > 0 ? P : MAXORD); i1++) {
      if (P == 0 && i1 >= p) break;
      const int ii = gidx((int)fr[0] - p + 1 + i1, A.n1);
      const long long v = __double2ll_rn((double)(th1[i1] * prod) * ORAC_QSCALE);
      if (v) atomicAdd(row + ii, (unsigned long long)v);
    }
  }
}

// Four lanes per atom, lane s taking the B-spline planes i3 = s, s+4, s+8
// of the p^3 grid points; the partial sums meet by shuffles.
constexpr int GATHER_LANES = 4;

template <int P>
__global__ void k_gather(const AtomArgs A) {
  pdl_enter();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int t = gt / GATHER_LANES, sub = gt % GATHER_LANES;
  const int p = P > 0 ? P : A.order;
  double st[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double dphi = 0.0;
  double fr[3] = {0, 0, 0};
  if (t < A.natom) frac_coord(A, t, fr);
  const bool active = t < A.natom && frac_ok(A, fr);
  float f1 = 0.f, f2 = 0.f, f3 = 0.f, phi = 0.f;
  if (active) {
    float th1[MAXORD], th2[MAXORD], th3[MAXORD], d1[MAXORD], d2[MAXORD], d3[MAXORD];
    bspline<P>((float)(fr[0] - (int)fr[0]), p, th1, d1);
    bspline<P>((float)(fr[1] - (int)fr[1]), p, th2, d2);
    bspline<P>((float)(fr[2] - (int)fr[2]), p, th3, d3);
    // the lane's planes i3 = sub, sub + GATHER_LANES, ...: the plane's
    // spline values picked from the arrays by constant indices, so every
    // lane of the warp runs its own plane at once (a loop over all planes
    // that skipped the others' ran each plane with a quarter of the lanes)
    constexpr int PP = P > 0 ? P : MAXORD;
#pragma unroll
    for (int c = 0; c < (PP + GATHER_LANES - 1) / GATHER_LANES; c++) {
      const int i3 = sub + c * GATHER_LANES;
      if (i3 >= p) break;
      float t3 = 0.f, dd3 = 0.f;
#pragma unroll
      for (int q = 0; q < PP; q++)
        if (q == i3) {
          t3 = th3[q];
          dd3 = d3[q];
        }
      const int kk = gidx((int)fr[2] - p + 1 + i3, A.n3);
#pragma unroll
      for (int i2 = 0; i2 < (P > 0 ? P : MAXORD); i2++) {
        if (P == 0 && i2 >= p) break;
        const int jj = gidx((int)fr[1] - p + 1 + i2, A.n2);
        const float* row = A.rg + ((size_t)kk * A.n2 + jj) * A.n1;
        float s1 = 0.f, s2 = 0.f, s3 = 0.f;
#pragma unroll
        for (int i1 = 0; i1 < (P > 0 ? P : MAXORD); i1++) {
          if (P == 0 && i1 >= p) break;
          const float qv = row[gidx((int)fr[0] - p + 1 + i1, A.n1)];
          s1 += d1[i1] * qv;
          s2 += th1[i1] * qv;
        }
        s3 = s2;
        phi += s2 * th2[i2] * t3;
        f1 += s1 * th2[i2] * t3;
        f2 += s2 * d2[i2] * t3;
        f3 += s3 * th2[i2] * dd3;
      }
    }
  }
#pragma unroll
  for (int o = 1; o < GATHER_LANES; o <<= 1) {
    f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    f2 += __shfl_xor_sync(0xffffffffu, f2, o);
    f3 += __shfl_xor_sync(0xffffffffu, f3, o);
    phi += __shfl_xor_sync(0xffffffffu, phi, o);
  }
  if (active && sub == 0) {
    const double qa = A.q[t];
    const double g1 = -A.n1 * qa * (double)f1, g2 = -A.n2 * qa * (double)f2, g3 = -A.n3 * qa * (double)f3;
    const double fx = A.r11 * g1 + A.r12 * g2 + A.r13 * g3;
    const double fy = A.r21 * g1 + A.r22 * g2 + A.r23 * g3;
    const double fz = A.r31 * g1 + A.r32 * g2 + A.r33 * g3;
    if (A.ffix) {  // fixed-point accumulator of the caller's RESPA level, which
                   // the shell pair kernel may be adding into at the same time
      atomicAdd(A.ffix + t, (unsigned long long)__double2ll_rn(fx * ORAC_FSCALE));
      atomicAdd(A.ffix + A.natom + t, (unsigned long long)__double2ll_rn(fy * ORAC_FSCALE));
      atomicAdd(A.ffix + 2 * A.natom + t, (unsigned long long)__double2ll_rn(fz * ORAC_FSCALE));
    } else {
      A.f[t] += fx;
      A.f[A.natom + t] += fy;
      A.f[2 * A.natom + t] += fz;
    }
    if (A.sxyz) {
      const int m = A.amol[t];
      const double sx = A.sxyz[t] - A.mol[m], sy = A.sxyz[A.natom + t] - A.mol[A.P + m],
                   sz = A.sxyz[2 * A.natom + t] - A.mol[2 * A.P + m];
      const double gx = sx * A.c11 + sy * A.c12 + sz * A.c13;
      const double gy = sy * A.c22 + sz * A.c23;
      const double gz = sz * A.c33;
      st[0] = -gx * fx;
      st[1] = -gy * fx;
      st[2] = -gz * fx;
      st[3] = -gx * fy;
      st[4] = -gy * fy;
      st[5] = -gz * fy;
      st[6] = -gx * fz;
      st[7] = -gy * fz;
      st[8] = -gz * fz;
    }
    if (A.dq) dphi = (double)phi * A.dq[t];
  }
  if (A.sxyz) block_reduce_add<9>(st, A.eout + 7);
  if (A.dq) block_reduce_add<1>(&dphi, A.edq);
}

void host_bspline(double w, int order, double* c, double* d) {
  c[order - 1] = 0.0;
  c[1] = w;
  c[0] = 1.0 - w;
  for (int k = 3; k <= order - 1; k++) {
    const double div = 1.0 / (k - 1);
    c[k - 1] = div * w * c[k - 2];
    for (int j = 1; j <= k - 2; j++) c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
    c[0] = div * (1 - w) * c[0];
  }
  d[0] = -c[0];
  for (int j = 2; j <= order; j++) d[j - 1] = c[j - 2] - c[j - 1];
  const int k = order;
  const double div = 1.0 / (k - 1);
  c[k - 1] = div * w * c[k - 2];
  for (int j = 1; j <= k - 2; j++) c[k - j - 1] = div * ((w + j) * c[k - j - 2] + (k - j - w) * c[k - j - 1]);
  c[0] = div * (1 - w) * c[0];
}

// load_bsp_moduli + DFTMOD (src/pme_fftw3.f90:165-230); twopi is 2 times a
// default-real (single precision) literal of pi in the reference.
void host_bsp_moduli(int nfft, int order, std::vector<float>& out) {
  std::vector<double> arr(order + 2), darr(order + 2), bsp(nfft + order + 2, 0.0), mod(nfft);
  host_bspline(0.0, order, arr.data(), darr.data());
  for (int i = 2; i <= order + 1 && i <= nfft; i++) bsp[i - 1] = arr[i - 2];
  const double twopi = 2.0 * (double)3.14159265358979323846f;
  for (int k = 1; k <= nfft; k++) {
    double s1 = 0, s2 = 0;
    for (int j = 1; j <= nfft; j++) {
      const double arg = twopi * (k - 1) * (j - 1) / nfft;
      s1 += bsp[j - 1] * cos(arg);
      s2 += bsp[j - 1] * sin(arg);
    }
    mod[k - 1] = s1 * s1 + s2 * s2;
  }
  for (int k = 1; k <= nfft; k++)
    if (mod[k - 1] < 1.0e-7) {
      const double lo = (k >= 2) ? mod[k - 2] : mod[nfft - 1];
      const double hi = (k <= nfft - 1) ? mod[k] : mod[0];
      mod[k - 1] = 0.5 * (lo + hi);
    }
  out.resize(nfft);
  for (int k = 0; k < nfft; k++) out[k] = (float)mod[k];
}

int upload_tw(orac_gpu_ctx* ctx, float2** dst, int n) {
  std::vector<float2> tw(n);
  const double pi = 4.0 * atan(1.0);
  for (int k = 0; k < n; k++) tw[k] = make_float2((float)cos(-2.0 * pi * k / n), (float)sin(-2.0 * pi * k / n));
  if (dev_alloc(ctx, dst, n)) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(*dst, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  return ORAC_OK;
}

// the builds of the spread and gather kernels for the common orders
using AtomKernel = void (*)(AtomArgs);
AtomKernel spread_kernel(int order) {
  return order == 4 ? k_spread<4> : order == 5 ? k_spread<5> : order == 6 ? k_spread<6> : order == 8 ? k_spread<8>
                                                                                                      : k_spread<0>;
}
AtomKernel gather_kernel(int order) {
  return order == 4 ? k_gather<4> : order == 5 ? k_gather<5> : order == 6 ? k_gather<6> : order == 8 ? k_gather<8>
                                                                                                      : k_gather<0>;
}

int lines_per_block(int n) {
  // few lines per block: the grids here are small (32^3-96^3), so many
  // small blocks spread a pass over all SMs
  // (2B + 1) lines of n complex values (two buffers of B lines and the
  // twiddles) in the 48 KB of shared memory a launch gets without opting in;
  // make_plan's axis limit keeps B >= 1 inside it
  int B = (49152 / (8 * n) - 1) / 2;
  if (B > 4) B = 4;
  if (B < 1) B = 1;
  return B;
}

}  // namespace

int pme_setup(orac_gpu_ctx* ctx, int n1, int n2, int n3, int order) {
  PmePlan& P = ctx->pme;
  if (order > MAXORD) return ctx_fail(ctx, ORAC_ERR_PARAM, "PME order %d > %d", order, MAXORD);
  FftPlan f;
  if (make_plan(n1, &f) || make_plan(n2, &f) || make_plan(n3, &f))
    return ctx_fail(ctx, ORAC_ERR_PARAM, "PME grid %dx%dx%d: sizes must factor into 2, 3, 5, 7", n1, n2, n3);
  if (P.n1 == n1 && P.n2 == n2 && P.n3 == n3 && P.order == order && P.qfix) return ORAC_OK;
  P.n1 = n1;
  P.n2 = n2;
  P.n3 = n3;
  P.order = order;
  P.h1 = n1 / 2 + 1;
  if (upload_tw(ctx, &P.tw1, n1) || upload_tw(ctx, &P.tw2, n2) || upload_tw(ctx, &P.tw3, n3)) return ORAC_ERR_CUDA;
  std::vector<float> b1, b2, b3;
  host_bsp_moduli(n1, order, b1);
  host_bsp_moduli(n2, order, b2);
  host_bsp_moduli(n3, order, b3);
  if (dev_alloc(ctx, &P.bsp1, n1) || dev_alloc(ctx, &P.bsp2, n2) || dev_alloc(ctx, &P.bsp3, n3)) return ORAC_ERR_CUDA;
  CK(cudaMemcpy(P.bsp1, b1.data(), sizeof(float) * n1, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.bsp2, b2.data(), sizeof(float) * n2, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(P.bsp3, b3.data(), sizeof(float) * n3, cudaMemcpyHostToDevice));
  const size_t ng = (size_t)n1 * n2 * n3;
  if (dev_alloc(ctx, &P.qfix, ng) || dev_alloc(ctx, &P.rgrid, ng) || dev_alloc(ctx, &P.cgrid, (size_t)P.h1 * n2 * n3))
    return ORAC_ERR_CUDA;
  return ORAC_OK;
}

int pme_run(orac_gpu_ctx* ctx, int natom, const double* d_cart, const double* d_q, const double* recip,
            double volume, double alpha, double* d_f, double* d_eout, const double* d_sxyz, const double* d_mol,
            unsigned long long* d_ffix, const double* d_dq, double* d_edq, float2* d_save,
            const float2* d_cross) {
  PmePlan& P = ctx->pme;
  if (!P.qfix) return ctx_fail(ctx, ORAC_ERR_STATE, "PME not set up");
  const int n1 = P.n1, n2 = P.n2, n3 = P.n3, h1 = P.h1;
  CK(cudaMemsetAsync(P.qfix, 0, sizeof(unsigned long long) * (size_t)n1 * n2 * n3, ctx->stream));
  CK(cudaMemsetAsync(d_eout, 0, sizeof(double) * 16, ctx->stream));
  AtomArgs A;
  memset(&A, 0, sizeof(A));
  A.natom = natom;
  A.order = P.order;
  A.n1 = n1;
  A.n2 = n2;
  A.n3 = n3;
  A.xyz = d_cart;
  A.q = d_q;
  A.r11 = recip[0];
  A.r21 = recip[1];
  A.r31 = recip[2];
  A.r12 = recip[3];
  A.r22 = recip[4];
  A.r32 = recip[5];
  A.r13 = recip[6];
  A.r23 = recip[7];
  A.r33 = recip[8];
  A.qfix = P.qfix;
  A.rg = P.rgrid;
  A.f = d_f;
  A.ffix = d_ffix;
  A.sxyz = d_sxyz;
  A.mol = d_mol;
  A.amol = ctx->d_amol;
  A.P = ctx->P;
  A.c11 = ctx->co[0];
  A.c12 = ctx->co[3];
  A.c13 = ctx->co[6];
  A.c22 = ctx->co[4];
  A.c23 = ctx->co[7];
  A.c33 = ctx->co[8];
  A.eout = d_eout;
  A.dq = d_edq ? d_dq : nullptr;
  A.edq = d_edq;
  const int nsp = natom * P.order;
  orac_launch(spread_kernel(P.order), (nsp + 255) / 256, 256, 0, ctx->stream, A);
  CKL();
  GridArgs G;
  memset(&G, 0, sizeof(G));
  G.n1 = n1;
  G.n2 = n2;
  G.n3 = n3;
  G.h1 = h1;
  G.qfix = P.qfix;
  G.cg = P.cgrid;
  G.rg = P.rgrid;
  G.bsp1 = P.bsp1;
  G.bsp2 = P.bsp2;
  G.bsp3 = P.bsp3;
  G.r11 = recip[0];
  G.r21 = recip[1];
  G.r31 = recip[2];
  G.r12 = recip[3];
  G.r22 = recip[4];
  G.r32 = recip[5];
  G.r13 = recip[6];
  G.r23 = recip[7];
  G.r33 = recip[8];
  const double pif = (double)3.14159265358979323846f;  // scalar_sum's single-precision pi
  G.fac = (float)(pif * pif / (alpha * alpha));
  G.pivol = (float)(pif * volume);
  G.rkcut2 = 0.25 * ctx->rkcut * ctx->rkcut / (pif * pif);
  G.eout = d_eout;
  G.save = d_save;
  G.cross = d_cross;
  int nb;
  size_t sm;
  {
    // x forward (r2c)
    make_plan(n1, &G.P);
    G.tw = P.tw1;
    G.B = lines_per_block(n1);
    nb = (n2 * n3 + G.B - 1) / G.B;
    sm = (2 * (size_t)G.B + 1) * n1 * sizeof(float2);
    orac_launch(k_fft<XF>, nb, FFT_THREADS, sm, ctx->stream, G);
    CKL();
    // y forward
    make_plan(n2, &G.P);
    G.tw = P.tw2;
    G.B = lines_per_block(n2);
    nb = n3 * ((h1 + G.B - 1) / G.B);
    sm = (2 * (size_t)G.B + 1) * n2 * sizeof(float2);
    orac_launch(k_fft<YF>, nb, FFT_THREADS, sm, ctx->stream, G);
    CKL();
  }
  // z forward + influence function + z inverse
  make_plan(n3, &G.P);
  G.tw = P.tw3;
  G.B = lines_per_block(n3);
  nb = n2 * ((h1 + G.B - 1) / G.B);
  sm = (2 * (size_t)G.B + 1) * n3 * sizeof(float2);
  orac_launch(k_fft<ZC>, nb, FFT_THREADS, sm, ctx->stream, G);
  CKL();
  // the energy alone (the second charge set of a non-equilibrium step's
  // work): no potential back on the grid, no gather
  if (d_cross || (!d_f && !d_ffix && !d_edq && !(d_sxyz && d_mol))) return ORAC_OK;
  {
    // y inverse
    make_plan(n2, &G.P);
    G.tw = P.tw2;
    G.B = lines_per_block(n2);
    nb = n3 * ((h1 + G.B - 1) / G.B);
    sm = (2 * (size_t)G.B + 1) * n2 * sizeof(float2);
    orac_launch(k_fft<YI>, nb, FFT_THREADS, sm, ctx->stream, G);
    CKL();
    // x inverse (c2r)
    make_plan(n1, &G.P);
    G.tw = P.tw1;
    G.B = lines_per_block(n1);
    nb = (n2 * n3 + G.B - 1) / G.B;
    sm = (2 * (size_t)G.B + 1) * n1 * sizeof(float2);
    orac_launch(k_fft<XI>, nb, FFT_THREADS, sm, ctx->stream, G);
    CKL();
  }
  orac_launch(gather_kernel(P.order), (GATHER_LANES * natom + 127) / 128, 128, 0, ctx->stream, A);
  CKL();
  return ORAC_OK;
}

// ---------------------------------------------------------------------------
// orac_gpu_pme_kspace_static: the SPME reciprocal sum of do_pmesh_kspace with
// no allocation at all.
//
// Some callers cannot allocate device memory: a host program that owns the
// whole HBM budget and hands libraries only buffers it carved out itself, a
// latency-bound serving loop that cannot take the device-wide
// synchronisation cudaMalloc / cudaFree imply, or a plugin whose host forbids
// allocation.  Such callers cannot create a context either (that allocates),
// so this entry point takes everything as arguments, reads and writes only
// the caller's device buffers, and keeps its working set -- charge grid,
// complex and real grids, twiddles, B-spline moduli, energy/virial sums -- in
// the fixed array below.  Every GPU that loads the library holds that array
// (ORAC_STATIC_PME_BYTES) until the process exits.
//
// Host code must never hand orac_static_pme_scratch itself to a kernel: on
// the host that name is a stand-in, not a device address.  The device address
// is looked up with cudaGetSymbolAddress, with the device current, on every
// call (static_scratch).
#define ORAC_STATIC_PME_BYTES (5u * 1024u * 1024u + 16u * 1024u)
static __device__ __align__(256) unsigned char orac_static_pme_scratch[ORAC_STATIC_PME_BYTES];

namespace {

constexpr int STATIC_MAX_AXIS = 256;             // points per grid axis
constexpr long long STATIC_MAX_POINTS = 262144;  // n1*n2*n3 (64^3)
constexpr int STATIC_MAX_DEVICES = 64;

std::mutex g_static_mu;
bool g_static_seen[STATIC_MAX_DEVICES];  // devices whose scratch address has been looked up once

struct SplineAt0 {
  double c[MAXORD + 2];
};

// Twiddles and |DFT(B-spline)|^2 moduli of the three axes (one block per
// axis), the same FP64 sums as upload_tw and host_bsp_moduli: only the order
// non-zero spline values enter the DFT, products and sums are kept unfused,
// and the small-modulus patch runs serially in index order like
// DFTMOD's loop (src/pme_fftw3.f90:202-230).
__global__ void k_static_tables(int n1, int n2, int n3, int order, SplineAt0 arr, float2* tw, float* bsp) {
  pdl_enter();
  __shared__ double mod[STATIC_MAX_AXIS];
  const int axis = blockIdx.x;
  const int n = axis == 0 ? n1 : (axis == 1 ? n2 : n3);
  float2* t = tw + axis * STATIC_MAX_AXIS;
  float* b = bsp + axis * STATIC_MAX_AXIS;
  const double pi = 3.14159265358979323846;
  const double twopi = 2.0 * (double)3.14159265358979323846f;  // single-precision pi, as DFTMOD
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    t[k] = make_float2((float)cos(-2.0 * pi * k / n), (float)sin(-2.0 * pi * k / n));
    double s1 = 0.0, s2 = 0.0;
    for (int j = 1; j <= order && j < n; j++) {
      const double arg = twopi * k * j / n;
      s1 = __dadd_rn(s1, __dmul_rn(arr.c[j - 1], cos(arg)));
      s2 = __dadd_rn(s2, __dmul_rn(arr.c[j - 1], sin(arg)));
    }
    mod[k] = __dadd_rn(__dmul_rn(s1, s1), __dmul_rn(s2, s2));
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < n; k++)
      if (mod[k] < 1.0e-7) mod[k] = 0.5 * ((k >= 1 ? mod[k - 1] : mod[n - 1]) + (k <= n - 2 ? mod[k + 1] : mod[0]));
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) b[k] = (float)mod[k];
}

// eer and the 3x3 column-major virial from the grid sums, as
// orac_gpu_do_pmesh_kspace finishes them on the host
__global__ void k_static_finish(const double* __restrict__ e, double* __restrict__ out) {
  pdl_enter();
  if (threadIdx.x != 0) return;
  out[0] = 0.5 * e[0];
  out[1] = 0.5 * e[1];
  out[2] = 0.5 * e[4];
  out[3] = 0.5 * e[5];
  out[4] = 0.5 * e[4];
  out[5] = 0.5 * e[2];
  out[6] = 0.5 * e[6];
  out[7] = 0.5 * e[5];
  out[8] = 0.5 * e[6];
  out[9] = 0.5 * e[3];
}

int static_fail(char* err, int err_len, int code, const char* fmt, ...) {
  if (err && err_len > 0) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, (size_t)err_len, fmt, ap);
    va_end(ap);
  }
  return code;
}

// Device address of the scratch array on device dev (which is current).
// Looked up on every call: if the process destroys the device's context and
// a new one is created (cudaDeviceReset, a primary-context reset by another
// library), the module is loaded again and the array may sit elsewhere, so a
// saved address could be stale.  The first lookup on a device may load the
// module, which must not happen inside a stream capture: such a first call
// is refused with ORAC_ERR_STATE.
int static_scratch(int dev, cudaStream_t st, unsigned char** out, char* err, int err_len) {
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_seen[dev]) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess)
      return static_fail(err, err_len, ORAC_ERR_STATE, "cudaStreamIsCapturing before the first call on device %d: %s",
                         dev, cudaGetErrorString(e));
    if (cs != cudaStreamCaptureStatusNone)
      return static_fail(err, err_len, ORAC_ERR_STATE,
                         "first call on device %d made while its stream is being captured: make one call on the "
                         "device before any capture",
                         dev);
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, orac_static_pme_scratch);
  if (e != cudaSuccess || !p)
    return static_fail(err, err_len, ORAC_ERR_CUDA, "cudaGetSymbolAddress of the SPME scratch on device %d: %s", dev,
                       cudaGetErrorString(e));
  g_static_seen[dev] = true;
  *out = (unsigned char*)p;
  return ORAC_OK;
}

size_t up256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int orac_gpu_pme_kspace_static(void* stream, int numatoms, const double* d_xyz, const double* d_charge,
                                          const double* recip, double volume, double ewald_coeff, double rkcut,
                                          int order, int nfft1, int nfft2, int nfft3, double* d_force,
                                          double* d_energy, char* err, int err_len) {
  if (err && err_len > 0) err[0] = '\0';
  if (numatoms <= 0) return static_fail(err, err_len, ORAC_ERR_PARAM, "numatoms = %d", numatoms);
  if (!d_xyz || !d_charge || !recip || !d_force || !d_energy)
    return static_fail(err, err_len, ORAC_ERR_PARAM, "null coordinate, charge, recip, force or energy pointer");
  if (order < 2 || order > MAXORD)
    return static_fail(err, err_len, ORAC_ERR_PARAM, "PME order %d outside 2..%d", order, MAXORD);
  if (!(volume > 0.0) || !(ewald_coeff > 0.0))
    return static_fail(err, err_len, ORAC_ERR_PARAM, "volume %g and ewald_coeff %g must be positive", volume,
                       ewald_coeff);
  const int dims[3] = {nfft1, nfft2, nfft3};
  FftPlan plan;
  for (int a = 0; a < 3; a++) {
    if (dims[a] > STATIC_MAX_AXIS)
      return static_fail(err, err_len, ORAC_ERR_CAPACITY,
                         "grid axis %d has %d points: the fixed scratch of orac_gpu_pme_kspace_static takes at most "
                         "%d per axis and %lld in all (64^3)",
                         a + 1, dims[a], STATIC_MAX_AXIS, STATIC_MAX_POINTS);
    if (dims[a] < order)
      return static_fail(err, err_len, ORAC_ERR_PARAM, "grid axis %d has %d points, fewer than the order %d", a + 1,
                         dims[a], order);
    if (make_plan(dims[a], &plan))
      return static_fail(err, err_len, ORAC_ERR_PARAM, "grid axis %d = %d does not factor into 2, 3, 5, 7", a + 1,
                         dims[a]);
  }
  const long long ng = (long long)nfft1 * nfft2 * nfft3;
  if (ng > STATIC_MAX_POINTS)
    return static_fail(err, err_len, ORAC_ERR_CAPACITY,
                       "grid %dx%dx%d has %lld points: the fixed scratch of orac_gpu_pme_kspace_static holds at "
                       "most %lld (64^3)",
                       nfft1, nfft2, nfft3, ng, STATIC_MAX_POINTS);
  const int h1 = nfft1 / 2 + 1;
  // scratch layout: sums | twiddles | moduli | charge grid | real grid | complex grid
  const size_t o_tw = 256;
  const size_t o_bsp = up256(o_tw + sizeof(float2) * 3 * STATIC_MAX_AXIS);
  const size_t o_q = up256(o_bsp + sizeof(float) * 3 * STATIC_MAX_AXIS);
  const size_t o_rg = up256(o_q + sizeof(unsigned long long) * (size_t)ng);
  const size_t o_cg = up256(o_rg + sizeof(float) * (size_t)ng);
  const size_t end = o_cg + sizeof(float2) * (size_t)h1 * nfft2 * nfft3;
  if (end > ORAC_STATIC_PME_BYTES)
    return static_fail(err, err_len, ORAC_ERR_CAPACITY, "grid %dx%dx%d needs %zu scratch bytes of %u", nfft1, nfft2,
                       nfft3, end, ORAC_STATIC_PME_BYTES);

  int dev = 0;
  cudaError_t ce = cudaGetDevice(&dev);
  if (ce != cudaSuccess)
    return static_fail(err, err_len, ORAC_ERR_NODEVICE, "cudaGetDevice: %s", cudaGetErrorString(ce));
  if (dev < 0 || dev >= STATIC_MAX_DEVICES)
    return static_fail(err, err_len, ORAC_ERR_PARAM, "device %d beyond the %d this entry point tracks", dev,
                       STATIC_MAX_DEVICES);
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* base = nullptr;
  if (int rc = static_scratch(dev, st, &base, err, err_len)) return rc;
  double* eout = (double*)base;
  float2* tw = (float2*)(base + o_tw);
  float* bsp = (float*)(base + o_bsp);
  unsigned long long* qfix = (unsigned long long*)(base + o_q);
  float* rgrid = (float*)(base + o_rg);
  float2* cgrid = (float2*)(base + o_cg);

  // what must start at zero: the fixed-point charge grid and the energy sums
  ce = cudaMemsetAsync(qfix, 0, sizeof(unsigned long long) * (size_t)ng, st);
  if (ce == cudaSuccess) ce = cudaMemsetAsync(eout, 0, sizeof(double) * 16, st);
  if (ce != cudaSuccess) return static_fail(err, err_len, ORAC_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(ce));

  SplineAt0 arr;
  double darr[MAXORD + 2];
  for (int k = 0; k < MAXORD + 2; k++) arr.c[k] = darr[k] = 0.0;
  host_bspline(0.0, order, arr.c, darr);
  orac_launch(k_static_tables, 3, 128, 0, st, nfft1, nfft2, nfft3, order, arr, tw, bsp);

  AtomArgs A;
  memset(&A, 0, sizeof(A));
  A.natom = numatoms;
  A.order = order;
  A.n1 = nfft1;
  A.n2 = nfft2;
  A.n3 = nfft3;
  A.xyz = d_xyz;
  A.q = d_charge;
  A.r11 = recip[0];
  A.r21 = recip[1];
  A.r31 = recip[2];
  A.r12 = recip[3];
  A.r22 = recip[4];
  A.r32 = recip[5];
  A.r13 = recip[6];
  A.r23 = recip[7];
  A.r33 = recip[8];
  A.qfix = qfix;
  A.rg = rgrid;
  A.f = d_force;
  A.eout = eout;
  const int nsp = numatoms * order;
  orac_launch(spread_kernel(order), (nsp + 255) / 256, 256, 0, st, A);

  GridArgs G;
  memset(&G, 0, sizeof(G));
  G.n1 = nfft1;
  G.n2 = nfft2;
  G.n3 = nfft3;
  G.h1 = h1;
  G.qfix = qfix;
  G.cg = cgrid;
  G.rg = rgrid;
  G.bsp1 = bsp;
  G.bsp2 = bsp + STATIC_MAX_AXIS;
  G.bsp3 = bsp + 2 * STATIC_MAX_AXIS;
  G.r11 = recip[0];
  G.r21 = recip[1];
  G.r31 = recip[2];
  G.r12 = recip[3];
  G.r22 = recip[4];
  G.r32 = recip[5];
  G.r13 = recip[6];
  G.r23 = recip[7];
  G.r33 = recip[8];
  const double pif = (double)3.14159265358979323846f;  // scalar_sum's single-precision pi
  const double rk = rkcut > 0.0 ? rkcut : 1e9;
  G.fac = (float)(pif * pif / (ewald_coeff * ewald_coeff));
  G.pivol = (float)(pif * volume);
  G.rkcut2 = 0.25 * rk * rk / (pif * pif);
  G.eout = eout;
  const float2* tws[3] = {tw, tw + STATIC_MAX_AXIS, tw + 2 * STATIC_MAX_AXIS};
  // x forward (r2c)
  make_plan(nfft1, &G.P);
  G.tw = tws[0];
  G.B = lines_per_block(nfft1);
  orac_launch(k_fft<XF>, (nfft2 * nfft3 + G.B - 1) / G.B, FFT_THREADS, (2 * (size_t)G.B + 1) * nfft1 * sizeof(float2), st, G);
  // y forward
  make_plan(nfft2, &G.P);
  G.tw = tws[1];
  G.B = lines_per_block(nfft2);
  orac_launch(k_fft<YF>, nfft3 * ((h1 + G.B - 1) / G.B), FFT_THREADS, (2 * (size_t)G.B + 1) * nfft2 * sizeof(float2), st, G);
  // z forward + influence function + z inverse
  make_plan(nfft3, &G.P);
  G.tw = tws[2];
  G.B = lines_per_block(nfft3);
  orac_launch(k_fft<ZC>, nfft2 * ((h1 + G.B - 1) / G.B), FFT_THREADS, (2 * (size_t)G.B + 1) * nfft3 * sizeof(float2), st, G);
  // y inverse
  make_plan(nfft2, &G.P);
  G.tw = tws[1];
  G.B = lines_per_block(nfft2);
  orac_launch(k_fft<YI>, nfft3 * ((h1 + G.B - 1) / G.B), FFT_THREADS, (2 * (size_t)G.B + 1) * nfft2 * sizeof(float2), st, G);
  // x inverse (c2r)
  make_plan(nfft1, &G.P);
  G.tw = tws[0];
  G.B = lines_per_block(nfft1);
  orac_launch(k_fft<XI>, (nfft2 * nfft3 + G.B - 1) / G.B, FFT_THREADS, (2 * (size_t)G.B + 1) * nfft1 * sizeof(float2), st, G);
  orac_launch(gather_kernel(order), (GATHER_LANES * numatoms + 127) / 128, 128, 0, st, A);
  orac_launch(k_static_finish, 1, 32, 0, st, eout, d_energy);
  ce = cudaGetLastError();
  if (ce != cudaSuccess) return static_fail(err, err_len, ORAC_ERR_CUDA, "SPME launch: %s", cudaGetErrorString(ce));
  return ORAC_OK;
}
