// fep.cu -- qfep's free-energy analysis (src/q6/qfep.f90:200-762) on the GPU.
//
// The per-point work (state totals, the ground-state energy, the energy gap,
// the exponential averages of Zwanzig, overlap sampling and BAR, the binned
// reaction free energies) runs in CUDA kernels over the energy records where
// they lie: a host copy for qb_fep_analyze, the engine's own record ring for
// qb_batch_fep.  The O(nfiles) running sums over windows follow on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "fep.hpp"
#include "qb.h"
#include "qsystem.hpp"

namespace qb {
void set_error(const std::string &m);

namespace {

constexpr int FEP_BLOCK = 256;
constexpr unsigned FULLMASK = 0xffffffffu;

#define FEP_CUDA(call)                                                                                   \
  do {                                                                                                   \
    cudaError_t e_ = (call);                                                                             \
    if (e_ != cudaSuccess) ::qb::fail(QB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Device view of one analysis.
struct FepDev {
  const double *E;            // energy records (see FepSource)
  const long long *foff;      // [nfiles]
  const int *npts;            // [nfiles]
  const int *pstart;          // [nfiles] first point of each file in V/VG/GAP
  int rs, ns, nfiles, nskip, gas, nbins, nmin;
  double rt;
  double alfa[QB_FEP_MAX_STATES], coeff[QB_FEP_MAX_STATES];
  double *lam;                // [nfiles*ns]
  double *V, *VG, *GAP;       // per point: shifted state totals, ground state, gap
  // EVB: r_xy of record p of file f at R[roff[f] + p*rrs]; Hij parameters [i*4+j]
  const double *R;
  const long long *roff;
  int rrs, nnoffd;
  double hA[QB_FEP_MAX_PAIRS], hmu[QB_FEP_MAX_PAIRS], heta[QB_FEP_MAX_PAIRS], hr0[QB_FEP_MAX_PAIRS];
  double *C1, *C2, *RX;       // per point: c1^2, c2^2 (two coupled states), r_xy
};

__device__ __forceinline__ const double *rec(const FepDev &D, int f, int p, int st) {
  return D.E + D.foff[f] + (long long)p * D.rs + st * QB_NEQ;
}

// A state's total of one record; with the gas option, the Q bonded, Q-Q and
// restraint terms only, summed in the reference's order (qfep.f90:259).
__device__ __forceinline__ double eq_total(const FepDev &D, const double *e) {
  if (D.gas > 0)
    return e[QB_EQ_BOND] + e[QB_EQ_ANGLE] + e[QB_EQ_TORSION] + e[QB_EQ_IMPROPER] + e[QB_EQ_QQ_EL] +
           e[QB_EQ_QQ_VDW] + e[QB_EQ_RESTRAINT];
  return e[QB_EQ_TOTAL];
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULLMASK, v, o);
  return v;
}

// Sum over the block, returned to every thread.
__device__ double block_sum_d(double v) {
  __shared__ double part[32];
  __shared__ double total;
  v = warp_sum_d(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  __syncthreads();
  if (lane == 0) part[w] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < nw; k++) t += part[k];
    total = t;
  }
  __syncthreads();
  return total;
}

// Lowest eigenvalue of a symmetric n x n matrix (n <= 4) by cyclic Jacobi
// rotations (Golub and Van Loan, Matrix Computations, 4th ed., 8.5.2-8.5.3):
// each rotation zeroes one off-diagonal element; sweeps until the
// off-diagonal mass is negligible against the matrix's.
__device__ double min_eigen(double (&a)[QB_FEP_MAX_STATES][QB_FEP_MAX_STATES], int n) {
  double fro = 0.0;
  for (int p = 0; p < n; p++)
    for (int q = 0; q < n; q++) fro += a[p][q] * a[p][q];
  for (int sweep = 0; sweep < 64; sweep++) {
    double off = 0.0;
    for (int p = 0; p < n; p++)
      for (int q = p + 1; q < n; q++) off += a[p][q] * a[p][q];
    if (off <= 1e-32 * fro) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        if (fabs(a[p][q]) < 1e-300) continue;
        const double tau = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
        const double c = 1.0 / sqrt(1.0 + t * t), s = t * c;
        for (int k = 0; k < n; k++) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; k++) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
      }
  }
  double m = a[0][0];
  for (int k = 1; k < n; k++) m = fmin(m, a[k][k]);
  return m;
}

// qfep's off-diagonal element of states i, j (0-based) at distance r: the
// parameters of (i, j), or of (j, i) where A(i, j) is 0 (qfep.f90:289-297).
__device__ __forceinline__ double evb_hij(const FepDev &D, int i, int j, double r) {
  int a = i * QB_FEP_MAX_STATES + j;
  if (D.hA[a] == 0.0) a = j * QB_FEP_MAX_STATES + i;
  const double d = r - D.hr0[a];
  return D.hA[a] * exp(-D.hmu[a] * d) * exp(-D.heta[a] * d * d);
}

// Per point (qfep.f90:257-322): shifted totals, ground state, energy gap;
// the file's lambdas from its first record.  With EVB coupling the ground
// state of two states is the lower root of the 2 x 2 secular equation, with
// the weights c1^2, c2^2 of the diabatic states; of more states, the lowest
// eigenvalue of the EVB matrix (qfep.f90:310-318).
__global__ void k_fep_values(FepDev D) {
  const int f = blockIdx.y;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= D.npts[f]) return;
  double tot[QB_FEP_MAX_STATES];
  for (int st = 0; st < D.ns; st++) {
    const double *e = rec(D, f, p, st);
    tot[st] = eq_total(D, e) + D.alfa[st];
    if (p == 0) D.lam[f * D.ns + st] = e[QB_EQ_LAMBDA];
  }
  const int q = D.pstart[f] + p;
  for (int st = 0; st < D.ns; st++) D.V[(size_t)q * D.ns + st] = tot[st];
  double vg, c1 = 0.0, c2 = 0.0, rx = 0.0;
  if (D.nnoffd > 0) rx = D.R[D.roff[f] + (long long)p * D.rrs];
  if (D.ns == 2) {
    const double hij = D.nnoffd > 0 ? evb_hij(D, 0, 1, rx) : 0.0;   // uncoupled without EVB
    vg = 0.5 * (tot[0] + tot[1]) - 0.5 * sqrt((tot[0] - tot[1]) * (tot[0] - tot[1]) + 4. * hij * hij);
    if (D.nnoffd > 0) {
      const double x = (vg - tot[0]) / hij;
      c1 = 1. / (1. + x * x);
      c2 = 1 - c1;
    }
  } else if (D.nnoffd > 0 && D.ns > 2) {
    double m[QB_FEP_MAX_STATES][QB_FEP_MAX_STATES];
    for (int i = 0; i < D.ns; i++) {
      m[i][i] = tot[i];
      for (int j = 0; j < i; j++) m[i][j] = m[j][i] = evb_hij(D, i, j, rx);   // the lower triangle
    }
    vg = min_eigen(m, D.ns);
  } else {
    vg = tot[0];
    for (int st = 1; st < D.ns; st++) vg = fmin(vg, tot[st]);
  }
  D.VG[q] = vg;
  D.C1[q] = c1;
  D.C2[q] = c2;
  D.RX[q] = rx;
  double g = 0.0;
  for (int st = 0; st < D.ns; st++) g = g + tot[st] * D.coeff[st];
  D.GAP[q] = g;
}

// Part 0 (qfep.f90:252-357): per file, the average of every component of
// every state over the points after nskip, summed in record order and scaled
// by the single-precision 1./(npts-nskip) of scale_ene.  One thread per
// (state, component).
__global__ void k_fep_part0(FepDev D, double *avEQ) {
  const int f = blockIdx.x, t = threadIdx.x;
  if (t >= D.ns * QB_NEQ) return;
  const int st = t / QB_NEQ, c = t % QB_NEQ;
  const int n = D.npts[f];
  double s = 0.0;
  for (int p = D.nskip; p < n; p++) {
    const double *e = rec(D, f, p, st);
    s += c == QB_EQ_TOTAL ? eq_total(D, e) : e[c];
  }
  const float k = 1.0f / (float)(n - D.nskip);
  avEQ[((size_t)f * D.ns + st) * QB_NEQ + c] = c == QB_EQ_LAMBDA ? D.lam[f * D.ns + st] : s * (double)k;
}

// Energy-gap range over the points after nskip, from qfep's starting values
// 999 / -999 (qfep.f90:200-201, 319-321).
__global__ void k_fep_gaprange(FepDev D, double *range) {
  __shared__ double smin[32], smax[32];
  double mn = 999., mx = -999.;
  for (int f = 0; f < D.nfiles; f++)
    for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
      const double g = D.GAP[D.pstart[f] + p];
      mn = fmin(mn, g);
      mx = fmax(mx, g);
    }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(FULLMASK, mn, o));
    mx = fmax(mx, __shfl_xor_sync(FULLMASK, mx, o));
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { smin[w] = mn; smax[w] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) { mn = fmin(mn, smin[k]); mx = fmax(mx, smax[k]); }
    range[0] = fmin(smin[0], mn);
    range[1] = fmax(smax[0], mx);
  }
}

// veff of point p of file g under the lambdas of file fl, summed over states
// in order as qfep does (veff = veff + lambda*v).
__device__ __forceinline__ double veff(const FepDev &D, int fl, int g, int p) {
  const double *v = D.V + (size_t)(D.pstart[g] + p) * D.ns;
  const double *l = D.lam + fl * D.ns;
  double s = 0.0;
  for (int st = 0; st < D.ns; st++) s = s + l[st] * v[st];
  return s;
}

struct PairOut {
  double *dgf, *dgr, *dgti, *dglu, *dgbar;
  int *its;
};

// One block per file f (entries f+1 of qfep's 1-based arrays):
//  TI (qfep.f90:448-469): <V2 - V1> over file f;
//  Zwanzig reverse (424-445): file f under lambda(f-1);
//  for the pair (f, f+1): Zwanzig forward (392-421), overlap sampling
//  (481-521) and BAR iterated from the overlap estimate to |change| <= 0.001
//  (524-578), at most QB_FEP_BAR_MAX_ITER rounds.
__global__ void k_fep_pairs(FepDev D, PairOut O) {
  const int f = blockIdx.x;
  const int nf = D.npts[f] - D.nskip;
  const double rt = D.rt;
  if (D.ns >= 2) {
    double s = 0.0;
    for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
      const double *v = D.V + (size_t)(D.pstart[f] + p) * D.ns;
      s += v[1] - v[0];
    }
    s = block_sum_d(s);
    if (threadIdx.x == 0) O.dgti[f + 1] = s / (double)nf;
  }
  if (f >= 1) {
    double s = 0.0;
    for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
      const double dv = veff(D, f - 1, f, p) - veff(D, f, f, p);
      s += exp(-dv / rt);
    }
    s = block_sum_d(s);
    if (threadIdx.x == 0) O.dgr[f + 1] = -rt * log(s / (double)nf);
  }
  if (f + 1 >= D.nfiles) return;
  const int g = f + 1;
  const int ng = D.npts[g] - D.nskip;
  double sf = 0.0, sof = 0.0, sob = 0.0;
  for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
    const double dv = veff(D, g, f, p) - veff(D, f, f, p);
    sf += exp(-dv / rt);
    sof += exp(-(dv / 2) / rt);
  }
  for (int p = D.nskip + threadIdx.x; p < D.npts[g]; p += blockDim.x) {
    const double dv = veff(D, g, g, p) - veff(D, f, g, p);
    sob += exp((dv / 2) / rt);
  }
  sf = block_sum_d(sf);
  sof = block_sum_d(sof);
  sob = block_sum_d(sob);
  const double dglu = -rt * log((sof / (double)nf) / (sob / (double)ng));
  if (threadIdx.x == 0) {
    O.dgf[f + 1] = -rt * log(sf / (double)nf);
    O.dglu[f + 1] = dglu;
  }
  // BAR: the sample-size ratios are single-precision quotients (qfep.f90:534-535)
  const double nfnr = (double)((float)nf / (float)ng), nrnf = (double)((float)ng / (float)nf);
  double konst = dglu, dg = dglu;
  int it = 0;
  bool done = false;
  while (!done && it < QB_FEP_BAR_MAX_ITER) {
    double a = 0.0, b = 0.0;
    for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
      const double dv = veff(D, g, f, p) - veff(D, f, f, p);
      a += 1 / (1 + (nfnr * exp((dv - konst) / rt)));
    }
    for (int p = D.nskip + threadIdx.x; p < D.npts[g]; p += blockDim.x) {
      const double dv = veff(D, g, g, p) - veff(D, f, g, p);
      b += 1 / (1 + (nrnf * exp((-dv + konst) / rt)));
    }
    a = block_sum_d(a) / (double)nf;
    b = block_sum_d(b) / (double)ng;
    dg = -rt * log((a / b) * exp(-konst / rt) * nfnr);
    const double fel = fabs(konst - dg);
    konst = dg;
    it++;
    done = !(fel > 0.001);
  }
  if (threadIdx.x == 0) {
    O.dgbar[f + 1] = dg;
    O.its[f + 1] = done ? it : -1;
  }
}

// int((gap - gapmin)/xint) + 1 (qfep.f90:628); a degenerate range (all gaps
// equal: 0/0) goes to bin 1, and the index stays within 0..nbins+1, where
// qfep's own result is undefined.
__device__ __forceinline__ int gap_bin(double gap, double gapmin, double xint, int nbins) {
  const double q = (gap - gapmin) / xint;
  int k;
  if (isnan(q)) k = 0;
  else if (q >= (double)(nbins + 1)) k = nbins + 1;
  else if (q <= -1.0) k = -1;
  else k = (int)q;
  return min(max(k + 1, 0), nbins + 1);
}

// Part 2 (qfep.f90:611-710), one block per file: per energy-gap bin the mean
// of V_i - veff and Vg - veff, then the exponential averages about them, and
// the diabatic and ground-state free energies dG(file) + ... for bins with at
// least nmin points.  Bin sums in shared memory.
__global__ void k_fep_bins(FepDev D, const double *range, const double *dG, double *part2) {
  extern __shared__ double bsm[];
  const int f = blockIdx.x, ns = D.ns, nb = D.nbins + 2;
  double *adv = bsm;                    // [nb*ns]
  double *adg = adv + nb * ns;          // [nb]
  double *sv = adg + nb;                // [nb*ns]
  double *sg = sv + nb * ns;            // [nb]
  double *ac1 = sg + nb, *ac2 = ac1 + nb, *arx = ac2 + nb;   // [nb] each: c1^2, c2^2, r_xy
  int *cnt = (int *)(arx + nb);         // [nb]
  for (int t = threadIdx.x; t < nb * ns; t += blockDim.x) { adv[t] = 0.0; sv[t] = 0.0; }
  for (int t = threadIdx.x; t < nb; t += blockDim.x) {
    adg[t] = 0.0; sg[t] = 0.0; cnt[t] = 0;
    ac1[t] = 0.0; ac2[t] = 0.0; arx[t] = 0.0;
  }
  __syncthreads();
  const double gapmin = range[0], xint = (range[1] - range[0]) / (double)D.nbins;
  const double rt = D.rt;
  for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
    const int q = D.pstart[f] + p;
    const int ib = gap_bin(D.GAP[q], gapmin, xint, D.nbins);
    const double ve = veff(D, f, f, p);
    for (int st = 0; st < ns; st++) atomicAdd(&adv[ib * ns + st], D.V[(size_t)q * ns + st] - ve);
    atomicAdd(&adg[ib], D.VG[q] - ve);
    atomicAdd(&ac1[ib], D.C1[q]);
    atomicAdd(&ac2[ib], D.C2[q]);
    if (D.nnoffd > 0) atomicAdd(&arx[ib], D.RX[q]);   // only the first r_xy (qfep.f90:643-644)
    atomicAdd(&cnt[ib], 1);
  }
  __syncthreads();
  for (int ib = 1 + threadIdx.x; ib <= D.nbins; ib += blockDim.x)
    if (cnt[ib] != 0) {
      for (int st = 0; st < ns; st++) adv[ib * ns + st] /= cnt[ib];
      adg[ib] /= cnt[ib];
      const double rn = (double)(float)cnt[ib];   // /real(nbinpts)
      ac1[ib] /= rn;
      ac2[ib] /= rn;
      arx[ib] /= rn;
    }
  __syncthreads();
  for (int p = D.nskip + threadIdx.x; p < D.npts[f]; p += blockDim.x) {
    const int q = D.pstart[f] + p;
    const int ib = gap_bin(D.GAP[q], gapmin, xint, D.nbins);
    const double ve = veff(D, f, f, p);
    for (int st = 0; st < ns; st++)
      atomicAdd(&sv[ib * ns + st], exp(-(D.V[(size_t)q * ns + st] - ve - adv[ib * ns + st]) / rt));
    atomicAdd(&sg[ib], exp(-(D.VG[q] - ve - adg[ib]) / rt));
  }
  __syncthreads();
  for (int ib = 1 + threadIdx.x; ib <= D.nbins; ib += blockDim.x) {
    double *r = part2 + ((size_t)f * nb + ib) * QB_FEP_PART2_W;
    for (int k = 0; k < QB_FEP_PART2_W; k++) r[k] = 0.0;
    r[0] = gapmin + (double)(float)ib * xint - xint / 2.;
    if (cnt[ib] < D.nmin) continue;
    const double n = (double)cnt[ib];
    const double dgf = dG[f + 1];
    r[1] = dgf + (-rt * log(sv[ib * ns + 0] / n) + adv[ib * ns + 0]);
    if (ns > 1) r[2] = dgf + (-rt * log(sv[ib * ns + 1] / n) + adv[ib * ns + 1]);
    r[3] = dgf + (-rt * log(sg[ib] / n) + adg[ib]);
    r[4] = n;
    r[5] = ac1[ib];
    r[6] = ac2[ib];
    r[7] = 1.0;
    r[8] = arx[ib];
  }
}

template <class T>
struct DevBuf {
  T *p = nullptr;
  explicit DevBuf(size_t n) { FEP_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T))); }
  ~DevBuf() { if (p) cudaFree(p); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

template <class T>
void put(T *dst, const std::vector<T> &src, cudaStream_t s) {
  if (!src.empty()) FEP_CUDA(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

template <class T>
void get(std::vector<T> &dst, const T *src, cudaStream_t s) {
  if (!dst.empty()) FEP_CUDA(cudaMemcpyAsync(dst.data(), src, dst.size() * sizeof(T), cudaMemcpyDeviceToHost, s));
}

template <class T>
void give(T *out, const std::vector<T> &v) {
  if (out) std::memcpy(out, v.data(), v.size() * sizeof(T));
}

}  // namespace

void fep_run(const FepSource &src, const qb_fep_params &p, int device, cudaStream_t stream, qb_fep_result *out) {
  const int nfiles = (int)src.npts.size(), ns = src.nstates;
  if (nfiles < 2) fail(QB_ERR_ARG, "the analysis needs at least two energy series");
  if (ns < 1 || ns > QB_FEP_MAX_STATES) fail(QB_ERR_ARG, "number of states must be 1..4");
  if (!(p.rt > 0.0)) fail(QB_ERR_ARG, "kT must be positive");
  if (p.nbins < 1 || p.nbins > QB_FEP_MAX_BINS) fail(QB_ERR_ARG, "number of gap bins must be 1..598");
  if (p.nskip < 0) fail(QB_ERR_ARG, "negative number of points to skip");
  for (int f = 0; f < nfiles; f++)
    if (src.npts[f] <= p.nskip)
      fail(QB_ERR_ARG, "number of data sets in series " + std::to_string(f + 1) +
                           " is less than number of points to skip");
  FEP_CUDA(cudaSetDevice(device));
  std::vector<int> pstart(nfiles);
  long long P = 0;
  int maxn = 0;
  for (int f = 0; f < nfiles; f++) { pstart[f] = (int)P; P += src.npts[f]; maxn = std::max(maxn, src.npts[f]); }
  const int nb = p.nbins + 2;

  DevBuf<long long> d_foff(nfiles);
  DevBuf<int> d_npts(nfiles), d_pstart(nfiles), d_its(nfiles + 2);
  DevBuf<double> d_lam((size_t)nfiles * ns), d_V((size_t)P * ns), d_VG(P), d_GAP(P);
  DevBuf<double> d_C1(P), d_C2(P), d_RX(P);
  DevBuf<long long> d_roff(nfiles);
  if (p.nnoffd < 0) fail(QB_ERR_ARG, "negative number of off-diagonal elements");
  if (p.nnoffd > 0 && (!src.rbase || (int)src.rfoff.size() != nfiles))
    fail(QB_ERR_ARG, "off-diagonal elements without r_xy values");
  DevBuf<double> d_av((size_t)nfiles * ns * QB_NEQ), d_range(2);
  DevBuf<double> d_dgf(nfiles + 2), d_dgr(nfiles + 2), d_dgti(nfiles + 2), d_dglu(nfiles + 2), d_dgbar(nfiles + 2);
  DevBuf<double> d_dG(nfiles + 2), d_part2((size_t)nfiles * nb * QB_FEP_PART2_W);
  put(d_foff.p, src.foff, stream);
  put(d_npts.p, src.npts, stream);
  put(d_pstart.p, pstart, stream);
  if (p.nnoffd > 0) put(d_roff.p, src.rfoff, stream);
  for (auto *b : {d_dgf.p, d_dgr.p, d_dgti.p, d_dglu.p, d_dgbar.p})
    FEP_CUDA(cudaMemsetAsync(b, 0, sizeof(double) * (nfiles + 2), stream));
  // k_fep_bins writes the rows of bins that hold points; the others must read
  // as empty (count 0), whatever the allocation held before
  FEP_CUDA(cudaMemsetAsync(d_part2.p, 0, sizeof(double) * (size_t)nfiles * nb * QB_FEP_PART2_W, stream));
  FEP_CUDA(cudaMemsetAsync(d_its.p, 0, sizeof(int) * (nfiles + 2), stream));

  FepDev D{};
  D.E = src.base; D.foff = d_foff.p; D.npts = d_npts.p; D.pstart = d_pstart.p;
  D.rs = src.rec_stride; D.ns = ns; D.nfiles = nfiles; D.nskip = p.nskip; D.gas = p.gas;
  D.nbins = p.nbins; D.nmin = p.nmin; D.rt = p.rt;
  for (int st = 0; st < QB_FEP_MAX_STATES; st++) {
    D.alfa[st] = st == 0 ? 0.0 : p.alfa[st];      // alfa(1)=0. (qfep.f90:264)
    D.coeff[st] = p.coeff[st];
  }
  D.lam = d_lam.p; D.V = d_V.p; D.VG = d_VG.p; D.GAP = d_GAP.p;
  D.C1 = d_C1.p; D.C2 = d_C2.p; D.RX = d_RX.p;
  D.nnoffd = p.nnoffd; D.R = src.rbase; D.roff = d_roff.p; D.rrs = src.r_stride;
  for (int k = 0; k < QB_FEP_MAX_PAIRS; k++) {
    D.hA[k] = p.evb_A[k]; D.hmu[k] = p.evb_mu[k]; D.heta[k] = p.evb_eta[k]; D.hr0[k] = p.evb_rxy0[k];
  }

  k_fep_values<<<dim3((maxn + FEP_BLOCK - 1) / FEP_BLOCK, nfiles), FEP_BLOCK, 0, stream>>>(D);
  k_fep_part0<<<nfiles, 64, 0, stream>>>(D, d_av.p);
  k_fep_gaprange<<<1, 1024, 0, stream>>>(D, d_range.p);
  PairOut O{d_dgf.p, d_dgr.p, d_dgti.p, d_dglu.p, d_dgbar.p, d_its.p};
  k_fep_pairs<<<nfiles, FEP_BLOCK, 0, stream>>>(D, O);
  FEP_CUDA(cudaGetLastError());

  std::vector<double> lam((size_t)nfiles * ns), av((size_t)nfiles * ns * QB_NEQ), range(2);
  std::vector<double> dgf(nfiles + 2), dgr(nfiles + 2), dgti(nfiles + 2), dglu(nfiles + 2), dgbar(nfiles + 2);
  std::vector<int> its(nfiles + 2);
  get(lam, d_lam.p, stream); get(av, d_av.p, stream); get(range, d_range.p, stream);
  get(dgf, d_dgf.p, stream); get(dgr, d_dgr.p, stream); get(dgti, d_dgti.p, stream);
  get(dglu, d_dglu.p, stream); get(dgbar, d_dgbar.p, stream); get(its, d_its.p, stream);
  FEP_CUDA(cudaStreamSynchronize(stream));

  // running sums over windows (qfep.f90:412-413, 436-437, 466-469, 511-512, 567, 586-589)
  std::vector<double> dgfsum(nfiles + 2, 0.0), dgrsum(nfiles + 2, 0.0), dG(nfiles + 2, 0.0);
  std::vector<double> dgtisum(nfiles + 2, 0.0), dglusum(nfiles + 2, 0.0), dgbarsum(nfiles + 2, 0.0);
  for (int i = 1; i <= nfiles - 1; i++) dgfsum[i + 1] = dgfsum[i] + dgf[i];
  for (int i = nfiles; i >= 2; i--) dgrsum[i - 1] = dgrsum[i] + dgr[i];
  for (int i = 2; i <= nfiles; i++) {
    const double dlam = lam[(size_t)(i - 2) * ns] - lam[(size_t)(i - 1) * ns];
    dgtisum[i] = dgtisum[i - 1] + (0.5 * (dgti[i - 1] + dgti[i]) * dlam);
  }
  for (int i = 1; i <= nfiles - 1; i++) dglusum[i + 1] = dglusum[i] + dglu[i];
  for (int i = 1; i <= nfiles - 1; i++) dgbarsum[i + 1] = dgbarsum[i] + dgbar[i];
  for (int i = 2; i <= nfiles; i++) dG[i] = dG[i - 1] + 0.5 * (dgf[i - 1] - dgr[i]);

  // Part 2 on the device, Part 3 (qfep.f90:721-745) from its rows in file order
  put(d_dG.p, dG, stream);
  const size_t smem = (size_t)nb * (2 * ns + 5) * sizeof(double) + (size_t)nb * sizeof(int);
  if (smem > 48 * 1024)
    FEP_CUDA(cudaFuncSetAttribute(k_fep_bins, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_fep_bins<<<nfiles, FEP_BLOCK, smem, stream>>>(D, d_range.p, d_dG.p, d_part2.p);
  FEP_CUDA(cudaGetLastError());
  std::vector<double> part2((size_t)nfiles * nb * QB_FEP_PART2_W);
  get(part2, d_part2.p, stream);
  FEP_CUDA(cudaStreamSynchronize(stream));

  std::vector<double> binsum((size_t)nb * 4, 0.0), part3((size_t)nb * QB_FEP_PART3_W, 0.0);
  std::vector<long long> ptsum(nb, 0);
  for (int f = 0; f < nfiles; f++)
    for (int ib = 1; ib <= p.nbins; ib++) {
      const double *r = &part2[((size_t)f * nb + ib) * QB_FEP_PART2_W];
      if (r[7] == 0.0) continue;
      const int n = (int)r[4];
      binsum[ib * 4 + 1] += r[5] * n;
      binsum[ib * 4 + 2] += r[6] * n;
      binsum[ib * 4 + 3] += r[8] * n;
      ptsum[ib] += n;
      binsum[ib * 4 + 0] += r[3] * n;
    }
  for (int ib = 1; ib <= p.nbins; ib++)
    if (ptsum[ib] >= p.nmin)
      for (int k = 0; k < 4; k++) binsum[ib * 4 + k] /= (double)(float)ptsum[ib];
  // the reference's minimum runs over its whole fixed-size bin array, zeros included
  double mn = 0.0;
  for (int ib = 1; ib <= p.nbins; ib++) mn = std::min(mn, binsum[ib * 4 + 0]);
  const double xint = (range[1] - range[0]) / (double)p.nbins;
  for (int ib = 1; ib <= p.nbins; ib++) {
    double *r = &part3[(size_t)ib * QB_FEP_PART3_W];
    r[0] = range[0] + (double)(float)ib * xint - xint / 2.;
    if (ptsum[ib] < p.nmin) continue;
    r[1] = binsum[ib * 4 + 0];
    r[2] = binsum[ib * 4 + 0] - mn;
    r[3] = (double)ptsum[ib];
    r[4] = binsum[ib * 4 + 1];
    r[5] = binsum[ib * 4 + 2];
    r[6] = binsum[ib * 4 + 3];
    r[7] = 1.0;
  }

  if (!out) return;
  give(out->lambda, lam);
  give(out->npts, src.npts);
  give(out->avEQ, av);
  give(out->dgf, dgf); give(out->dgfsum, dgfsum);
  give(out->dgr, dgr); give(out->dgrsum, dgrsum);
  give(out->dG, dG);
  give(out->dgti, dgti); give(out->dgtisum, dgtisum);
  give(out->dglu, dglu); give(out->dglusum, dglusum);
  give(out->dgbar, dgbar); give(out->dgbarsum, dgbarsum);
  give(out->bar_iterations, its);
  give(out->gap_range, range);
  give(out->part2, part2);
  give(out->part3, part3);
}

}  // namespace qb

extern "C" int qb_fep_analyze(const double *energies, const int *npts, int nfiles, int nstates,
                              const qb_fep_params *p, int device, qb_fep_result *out) {
  if (!energies || !npts || !p || nfiles < 1) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  try {
    qb::FepSource src;
    src.nstates = nstates;
    src.rec_stride = nstates * QB_NEQ;
    long long total = 0;
    for (int f = 0; f < nfiles; f++) {
      if (npts[f] < 0) qb::fail(QB_ERR_ARG, "negative record count");
      src.foff.push_back(total * src.rec_stride);
      src.npts.push_back(npts[f]);
      total += npts[f];
    }
    if (nstates < 1 || nstates > QB_FEP_MAX_STATES) qb::fail(QB_ERR_ARG, "number of states must be 1..4");
    if (p->nnoffd > 0 && !p->rxy) qb::fail(QB_ERR_ARG, "off-diagonal elements without r_xy values");
    FEP_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    FEP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    double *dE = nullptr;
    // the records, then (EVB) every record's r_xy
    const long long nE = total * src.rec_stride, nR = p->nnoffd > 0 ? total : 0;
    cudaError_t e = cudaMalloc(&dE, sizeof(double) * std::max<long long>(nE + nR, 1));
    if (e != cudaSuccess) { cudaStreamDestroy(s); qb::fail(QB_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); }
    try {
      FEP_CUDA(cudaMemcpyAsync(dE, energies, sizeof(double) * nE, cudaMemcpyHostToDevice, s));
      src.base = dE;
      if (nR > 0) {
        FEP_CUDA(cudaMemcpyAsync(dE + nE, p->rxy, sizeof(double) * nR, cudaMemcpyHostToDevice, s));
        src.rbase = dE + nE;
        src.r_stride = 1;
        long long off = 0;
        for (int f = 0; f < nfiles; f++) { src.rfoff.push_back(off); off += npts[f]; }
      }
      qb::fep_run(src, *p, device, s, out);
    } catch (...) {
      cudaStreamSynchronize(s);
      cudaFree(dE);
      cudaStreamDestroy(s);
      throw;
    }
    cudaStreamSynchronize(s);
    cudaFree(dE);
    cudaStreamDestroy(s);
    return QB_OK;
  } catch (const qb::Error &e) {
    qb::set_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    qb::set_error(e.what());
    return QB_ERR_STATE;
  }
}
