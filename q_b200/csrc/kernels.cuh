// kernels.cuh -- per-step device kernels of the Q MD step (sm_100a).
//
// One launch covers every system of a batch.  Most kernels use a 2-D grid:
// blockIdx.y selects the system and blockIdx.x/threadIdx stride over that
// system's items, so each block reduces energies of one system only.
// Each kernel names the reference routine (src/q6/md.f90) it restates.
#pragma once
#include <cuda_runtime.h>

#include <type_traits>

#include "engine.cuh"

namespace qb {

constexpr unsigned FULL = 0xffffffffu;
constexpr float kBoltzF = 0.001986f;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

// Reduce v over the warp and add it to *dst once (lane 0).  All 32 lanes of
// the warp must call it.
__device__ __forceinline__ void warp_add(double *dst, double v) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

__device__ __forceinline__ double3 ld3(const double4 *p, int g) {
  double4 a = p[g];
  return make_double3(a.x, a.y, a.z);
}

__device__ __forceinline__ void atomic_add3(double4 *d, int g, double fx, double fy, double fz) {
  atomicAdd(&d[g].x, fx);
  atomicAdd(&d[g].y, fy);
  atomicAdd(&d[g].z, fz);
}

__device__ __forceinline__ void set_status(SysState *st, int code) { atomicCAS(&st->status, 0, code); }

__device__ __forceinline__ double dev_pi() { return (double)(4.0f * atanf(1.0f)); }

// ------------------------------------------------------------ periodic box

// Edge lengths and their inverses of system s's box.  The nearest image of a
// displacement d along an edge is d - L nint(d / L), written as the reference
// writes it, boxlength * nint(d * inv_boxl) (md.f90:5352-5354, 10513-10519);
// nint rounds halves away from zero, as round() does.
struct BoxD { double L[3], iL[3]; };

__device__ __forceinline__ BoxD box_of(const DevPtrs &P, int s) {
  const SysState &st = P.st[s];
  BoxD b;
#pragma unroll
  for (int k = 0; k < 3; k++) { b.L[k] = st.boxl[k]; b.iL[k] = st.iboxl[k]; }
  return b;
}

// the lattice vector L nint(d / L) that brings d to its nearest image
__device__ __forceinline__ double3 image_shift(const BoxD &b, double dx, double dy, double dz) {
  return make_double3(b.L[0] * round(dx * b.iL[0]), b.L[1] * round(dy * b.iL[1]), b.L[2] * round(dz * b.iL[2]));
}

__device__ __forceinline__ void min_image(const BoxD &b, double &dx, double &dy, double &dz) {
  const double3 t = image_shift(b, dx, dy, dz);
  dx -= t.x; dy -= t.y; dz -= t.z;
}

// the switching atom of an atom's charge group
__device__ __forceinline__ int switch_of(const DevPtrs &P, int a) { return P.cg_sw[P.cgp[a]]; }

// ------------------------------------------------------------------ lists

// Lists of system s are rebuilt at steps that are multiples of its non_bond
// interval (md.f90:4005), or on request (the post-loop rebuild, md.f90:4186).
// force 2: the systems in a volume move (MC_volume rebuilds their LRF and
// pair lists for the trial box, md.f90:15734-15744).
__device__ __forceinline__ bool list_due(const DevPtrs &P, int s, int force) {
  if (force == 2) return P.st[s].mc != 0;
  return force || (P.st[s].istep % P.sys[s].NB) == 0;
}

// cgp_centers (md.f90:1000): group centres, multipoles zeroed.
__global__ void k_cgp_centers(DevPtrs P, int force) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= P.ncgp_tot) return;
  if (!list_due(P, P.cg_sys[g], force)) return;
  double c[3] = {0, 0, 0};
  int f = P.cg_first[g], l = P.cg_last[g];
  for (int a = f; a <= l; a++) {
    double3 xa = ld3(P.x, P.cg_atoms[a]);
    c[0] += xa.x; c[1] += xa.y; c[2] += xa.z;
  }
  double n = (double)(float)(l - f + 1);
  double *L = P.lrf + (size_t)g * LRF_STRIDE;
  for (int k = 0; k < 3; k++) L[k] = c[k] / n;
  for (int k = 3; k < LRF_STRIDE - 1; k++) L[k] = 0.0;
  // radius: bounds every atom pair of two groups by their centres (the
  // any-atom cut-off tests of iuse_switch_atom 0 skip far groups with it)
  double rmax = 0.0;
  for (int a = f; a <= l; a++) {
    double3 xa = ld3(P.x, P.cg_atoms[a]);
    double dx = xa.x - L[0], dy = xa.y - L[1], dz = xa.z - L[2];
    rmax = fmax(rmax, sqrt(dx * dx + dy * dy + dz * dz));
  }
  L[LRF_STRIDE - 1] = rmax;
}

// The any-atom cut-off tests of iuse_switch_atom 0 (nbpplis2_lrf md.f90:4955,
// nbpwlis2_lrf 6500, nbqplis2 7700), FP64 as the reference.
// Solute group pair: inside when any atom pair of the two groups is within
// rc2; *last receives the squared distance of the last pair computed (the two
// groups' last atoms when none is inside), which the reference then tests
// against RcLRF.
__device__ __forceinline__ bool groups_inside_any(const DevPtrs &P, int gi, int gj, double rc2, double *last) {
  double r2 = 0.0;
  for (int ia = P.cg_first[gi]; ia <= P.cg_last[gi]; ia++) {
    const double3 xi = ld3(P.x, P.cg_atoms[ia]);
    for (int ja = P.cg_first[gj]; ja <= P.cg_last[gj]; ja++) {
      const double3 xj = ld3(P.x, P.cg_atoms[ja]);
      const double dx = xi.x - xj.x, dy = xi.y - xj.y, dz = xi.z - xj.z;
      r2 = dx * dx + dy * dy + dz * dz;
      if (r2 <= rc2) { *last = r2; return true; }
    }
  }
  *last = r2;
  return false;
}

// Solute group and a point (a water O or the solute centre): inside when any
// atom of the group is within rc2 of it; *last as above.
__device__ __forceinline__ bool group_point_inside_any(const DevPtrs &P, int gi, double3 p, double rc2, double *last) {
  double r2 = 0.0;
  for (int ia = P.cg_first[gi]; ia <= P.cg_last[gi]; ia++) {
    const double3 xi = ld3(P.x, P.cg_atoms[ia]);
    const double dx = xi.x - p.x, dy = xi.y - p.y, dz = xi.z - p.z;
    r2 = dx * dx + dy * dy + dz * dz;
    if (r2 <= rc2) { *last = r2; return true; }
  }
  *last = r2;
  return false;
}

// Bounds from the groups' centres and radii (the LRF records, written by
// k_cgp_centers before the list kernels): -1 when no atom pair can be within
// the cut-off, +1 when every atom pair is, 0 when only the atoms can tell.  The
// margin keeps pairs near the cut-off for the exact FP64 atom test.
__device__ __forceinline__ int groups_reach(const DevPtrs &P, int gi, int gj, double rc2) {
  const double *Li = P.lrf + (size_t)gi * LRF_STRIDE, *Lj = P.lrf + (size_t)gj * LRF_STRIDE;
  const double dx = Li[0] - Lj[0], dy = Li[1] - Lj[1], dz = Li[2] - Lj[2];
  const double dc = sqrt(dx * dx + dy * dy + dz * dz), rr = Li[LRF_STRIDE - 1] + Lj[LRF_STRIDE - 1];
  const double rc = sqrt(rc2);
  if (dc - rr > rc + 1e-6) return -1;
  if (dc + rr < rc - 1e-6) return 1;
  return 0;
}

__device__ __forceinline__ int group_point_reach(const DevPtrs &P, int gi, double3 p, double rc2) {
  const double *Li = P.lrf + (size_t)gi * LRF_STRIDE;
  const double dx = Li[0] - p.x, dy = Li[1] - p.y, dz = Li[2] - p.z;
  const double dc = sqrt(dx * dx + dy * dy + dz * dz), rr = Li[LRF_STRIDE - 1];
  const double rc = sqrt(rc2);
  if (dc - rr > rc + 1e-6) return -1;
  if (dc + rr < rc - 1e-6) return 1;
  return 0;
}

// Near/far test of an LRF gather pair (target group g, source group h) under
// iuse_switch_atom 0, when one of them is a solute group: true when the pair
// takes part in the LRF (outside the any-atom cut-off, last pair within
// RcLRF).  Groups whose centres are farther apart than the cut-off plus both
// radii (with a margin) are outside without the atom loop.
__device__ __forceinline__ bool lrf_window_any(const DevPtrs &P, const SysDev &S, int g, bool g_sol, int h, bool h_sol,
                                               double rc2) {
  const double *Lg = P.lrf + (size_t)g * LRF_STRIDE, *Lh = P.lrf + (size_t)h * LRF_STRIDE;
  const double dx = Lg[0] - Lh[0], dy = Lg[1] - Lh[1], dz = Lg[2] - Lh[2];
  const double dc = sqrt(dx * dx + dy * dy + dz * dz);
  const bool far = dc - Lg[LRF_STRIDE - 1] - Lh[LRF_STRIDE - 1] > sqrt(rc2) + 1e-6;
  double last;
  bool inside;
  if (g_sol && h_sol) {
    if (far) {
      const double3 a = ld3(P.x, P.cg_atoms[P.cg_last[g]]), b = ld3(P.x, P.cg_atoms[P.cg_last[h]]);
      last = (a.x - b.x) * (a.x - b.x) + (a.y - b.y) * (a.y - b.y) + (a.z - b.z) * (a.z - b.z);
      inside = false;
    } else {
      inside = groups_inside_any(P, g, h, rc2, &last);
    }
  } else {
    // solute group and water: the group's atoms against the water O
    const int gs = g_sol ? g : h, gw = g_sol ? h : g;
    const double3 o = ld3(P.x, P.cg_sw[gw]);
    if (far) {
      const double3 a = ld3(P.x, P.cg_atoms[P.cg_last[gs]]);
      last = (a.x - o.x) * (a.x - o.x) + (a.y - o.y) * (a.y - o.y) + (a.z - o.z) * (a.z - o.z);
      inside = false;
    } else {
      inside = group_point_inside_any(P, gs, o, rc2, &last);
    }
  }
  return !inside && last <= S.RcLRF2;
}

// Multipole contribution of charge q at offset (dx,dy,dz) from a group centre
// (md.f90:5581-5636), accumulated in the symmetric form m[20] = phi0,
// phi1[x,y,z], phi2[xx,xy,xz,yy,yz,zz], phi3[xxx,xxy,xxz,xyy,xyz,xzz,yyy,yyz,
// yzz,zzz]: the reference's 9 and 27 components are copies of these.
// 1/sqrt(v) on the MUFU unit (rsqrt.approx.ftz.f32, <= 2 ulp); the squared
// distances it is used on are never denormal.
__device__ __forceinline__ float rsqrt_ftz(float v) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(v));
  return r;
}

__device__ __forceinline__ float rsq(float v) { return rsqrt_ftz(v); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ double rsq(double v) { return rsqrt(v); }

template <class R>
__device__ __forceinline__ void lrf_accumulate(R *m, R q, R dx, R dy, R dz) {
  R r2 = dx * dx + dy * dy + dz * dz;
  R rinv = rsq(r2), ri2 = rinv * rinv;
  R f0 = q * rinv * ri2;              // q / r^3
  m[0] += f0 * r2;
  m[1] -= f0 * dx; m[2] -= f0 * dy; m[3] -= f0 * dz;
  R f1 = R(3) * f0 * ri2;
  R f1x = f1 * dx, f1y = f1 * dy, f1z = f1 * dz;
  m[4] += f1x * dx - f0; m[5] += f1x * dy; m[6] += f1x * dz;
  m[7] += f1y * dy - f0; m[8] += f1y * dz; m[9] += f1z * dz - f0;
  R f2 = -f1 * ri2;
  R x5 = R(5) * dx, y5 = R(5) * dy, z5 = R(5) * dz;
  R xx = x5 * dx, yy = y5 * dy, zz = z5 * dz, xy = x5 * dy;
  m[10] += f2 * (xx * dx - R(3) * r2 * dx);
  m[11] += f2 * (xx * dy - r2 * dy);
  m[12] += f2 * (xx * dz - r2 * dz);
  m[13] += f2 * (yy * dx - r2 * dx);
  m[14] += f2 * (xy * dz);
  m[15] += f2 * (zz * dx - r2 * dx);
  m[16] += f2 * (yy * dy - R(3) * r2 * dy);
  m[17] += f2 * (yy * dz - r2 * dz);
  m[18] += f2 * (zz * dy - r2 * dy);
  m[19] += f2 * (zz * dz - R(3) * r2 * dz);
}

// The same sums with the diagonal terms of phi2 and phi3 factored out:
// m[0..19] as above without them, plus t[0] = sum f0 and t[1..3] = sum
// f2*r2*d; lrf_fold applies them once at the end (phi2_aa -= t0,
// phi3_aab -= t_b for a != b, phi3_aaa -= 3 t_a).  22 fewer operations per
// charge; used by the mixed-precision gather.
__device__ __forceinline__ void lrf_accumulate_split(float *m, float *t, float q, float dx, float dy, float dz) {
  float r2 = dx * dx + dy * dy + dz * dz;
  float rinv = rsqrt_ftz(r2), ri2 = rinv * rinv;
  float f0 = q * rinv * ri2;
  m[0] = fmaf(f0, r2, m[0]);
  m[1] = fmaf(-f0, dx, m[1]); m[2] = fmaf(-f0, dy, m[2]); m[3] = fmaf(-f0, dz, m[3]);
  t[0] += f0;
  float f1 = 3.f * f0 * ri2;
  float ax = f1 * dx, ay = f1 * dy, az = f1 * dz;
  m[4] = fmaf(ax, dx, m[4]); m[5] = fmaf(ax, dy, m[5]); m[6] = fmaf(ax, dz, m[6]);
  m[7] = fmaf(ay, dy, m[7]); m[8] = fmaf(ay, dz, m[8]); m[9] = fmaf(az, dz, m[9]);
  float f2 = -f1 * ri2;
  float w = f2 * r2;
  t[1] = fmaf(w, dx, t[1]); t[2] = fmaf(w, dy, t[2]); t[3] = fmaf(w, dz, t[3]);
  float u = 5.f * f2;
  float px = u * dx, py = u * dy;
  float qxx = px * dx, qxy = px * dy, qxz = px * dz, qyy = py * dy, qyz = py * dz, qzz = u * dz * dz;
  m[10] = fmaf(qxx, dx, m[10]); m[11] = fmaf(qxx, dy, m[11]); m[12] = fmaf(qxx, dz, m[12]);
  m[13] = fmaf(qxy, dy, m[13]); m[14] = fmaf(qxy, dz, m[14]); m[15] = fmaf(qxz, dz, m[15]);
  m[16] = fmaf(qyy, dy, m[16]); m[17] = fmaf(qyy, dz, m[17]); m[18] = fmaf(qyz, dz, m[18]);
  m[19] = fmaf(qzz, dz, m[19]);
}

__device__ __forceinline__ void lrf_fold(double *m, const double *t) {
  m[4] -= t[0]; m[7] -= t[0]; m[9] -= t[0];
  m[10] -= 3. * t[1]; m[11] -= t[2]; m[12] -= t[3];
  m[13] -= t[1]; m[15] -= t[1];
  m[16] -= 3. * t[2]; m[17] -= t[3]; m[18] -= t[2];
  m[19] -= 3. * t[3];
}

// LRF multipoles of every charge group, gathered (nbpplist_lrf 5448,
// nbpwlist_lrf 6864, nbwwlist_lrf 8370).  A group g receives the charges of
// every group h whose switching atoms lie beyond the pair's cut-off but within
// RcLRF (both switching atoms inside the sphere; solute Q atoms carry no
// charge here).  The reference visits each unordered pair once and adds to
// both groups; the gather adds the same contributions.
//
// One thread per group g, blockIdx.y = system.  The system's groups are swept
// in tiles (consecutive groups, at most LRF_TILE_G groups and LRF_TILE_A
// atoms, boundaries precomputed on the host): a tile's switching atoms and
// atom positions/charges are staged in shared memory and read as broadcasts.
// The group-pair window test is FP64 in both precisions.  Mixed precision:
// atom offsets from the group centre in FP32 (positions relative to the
// sphere centre, |offset| >= ~7 A here), each tile summed in FP32 and added to
// FP64 totals.
constexpr int LRF_TILE_G = 128, LRF_TILE_A = 512, LRF_BLOCK = 128;
constexpr int LRF_TILES_PER_BLOCK = 4;   // default source tiles per block (P.lrf_tpb); larger systems use more blocks

template <bool MIXED>
__global__ void __launch_bounds__(LRF_BLOCK, MIXED ? 8 : 5) k_lrf_gather(DevPtrs P, int force) {
  using R = typename std::conditional<MIXED, float, double>::type;
  using R4 = typename std::conditional<MIXED, float4, double4>::type;
  int s = blockIdx.y;
  if (!list_due(P, s, force)) return;
  const SysDev &S = P.sys[s];
  if (!S.use_lrf) return;
  // block -> (chunk of target groups, range of source tiles)
  const int tpb = P.lrf_tpb;
  const int hsplit = (S.nlrft + tpb - 1) / tpb;
  const int gchunk = blockIdx.x / max(hsplit, 1), hpart = blockIdx.x % max(hsplit, 1);
  if (hsplit == 0 || gchunk * LRF_BLOCK >= S.ncgp) return;
  const int t0 = hpart * tpb, t1 = min(t0 + tpb, S.nlrft);
  __shared__ double4 hsw[LRF_TILE_G];      // switching atom; w: -1 excluded, 1 solute, 0 water
  __shared__ int2 hrange[LRF_TILE_G];      // first atom slot, atom count
  __shared__ R4 hat[LRF_TILE_A];           // atom position (mixed: from the sphere centre), charge
  int gl = gchunk * LRF_BLOCK + threadIdx.x;
  int g = S.coff + gl;
  bool active = gl < S.ncgp;
  double cx = 0, cy = 0, cz = 0;
  double3 xs = make_double3(0, 0, 0);
  if (active) {
    int swg = P.cg_sw[g];
    active = !(P.flags[swg] & F_EXCL);
    const double *L = P.lrf + (size_t)g * LRF_STRIDE;
    cx = L[0]; cy = L[1]; cz = L[2];
    xs = ld3(P.x, swg);
  }
  const double ox = MIXED ? S.origin[0] : 0.0, oy = MIXED ? S.origin[1] : 0.0, oz = MIXED ? S.origin[2] : 0.0;
  const R ccx = (R)(cx - ox), ccy = (R)(cy - oy), ccz = (R)(cz - oz);
  const bool g_sol = gl < S.ncgp_sol;
  // periodic box: pair windows on the switching atoms' nearest image; a
  // source group's charges enter at the image nearest the target centre
  // (nbpplist_box_lrf md.f90:5751-5849, nbpwlist_box_lrf 7111-7245,
  // nbwwlist_box_lrf 8601-8694)
  const bool box = S.pbc != 0;
  const BoxD bx = box_of(P, s);
  // FP64 totals: registers (FP64 path) or this thread's column in shared memory (mixed)
  __shared__ double mtot[MIXED ? 24 : 1][MIXED ? LRF_BLOCK : 1];
  double m[MIXED ? 1 : 20];
  R mt[20];
  float tt[4];
  if (MIXED) {
#pragma unroll
    for (int k = 0; k < 24; k++) mtot[k][threadIdx.x] = 0.0;
  } else {
#pragma unroll
    for (int k = 0; k < 20; k++) m[k] = 0.0;
  }
  for (int t = t0; t < t1; t++) {
    int2 tile = P.lrft[S.lrft_off + t];
    int nh = tile.y - tile.x;
    int a0 = P.cg_first[S.coff + tile.x];
    int na = P.cg_last[S.coff + tile.y - 1] - a0 + 1;
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += LRF_BLOCK) {
      int h = S.coff + tile.x + i;
      int sw = P.cg_sw[h];
      double3 p = ld3(P.x, sw);
      double w = (P.flags[sw] & F_EXCL) ? -1.0 : (tile.x + i < S.ncgp_sol ? 1.0 : 0.0);
      hsw[i] = make_double4(p.x, p.y, p.z, w);
      hrange[i] = make_int2(P.cg_first[h] - a0, P.cg_last[h] - P.cg_first[h] + 1);
    }
    for (int i = threadIdx.x; i < na; i += LRF_BLOCK) {
      int at = P.cg_atoms[a0 + i];
      double4 p = P.x[at];
      bool qsol = (at - S.aoff) < S.nsol && P.iq[at] >= 0;
      R4 v;
      v.x = (R)(p.x - ox); v.y = (R)(p.y - oy); v.z = (R)(p.z - oz);
      v.w = qsol ? R(0) : (R)P.crg[at];
      hat[i] = v;
    }
    __syncthreads();
    if (active) {
      if (MIXED) {
#pragma unroll
        for (int k = 0; k < 20; k++) mt[k] = R(0);
#pragma unroll
        for (int k = 0; k < 4; k++) tt[k] = 0.f;
      }
      for (int i = 0; i < nh; i++) {
        double4 hs = hsw[i];
        if (hs.w < 0.0 || tile.x + i == gl) continue;
        double rc2 = (g_sol && hs.w > 0.0) ? S.Rcpp2 : ((g_sol || hs.w > 0.0) ? S.Rcpw2 : S.Rcww2);
        if (!S.switch_atoms && (g_sol || hs.w > 0.0)) {
          if (!lrf_window_any(P, S, g, g_sol, S.coff + tile.x + i, hs.w > 0.0, rc2)) continue;
        } else {
          double dx = xs.x - hs.x, dy = xs.y - hs.y, dz = xs.z - hs.z;
          if (box) min_image(bx, dx, dy, dz);
          double r2 = dx * dx + dy * dy + dz * dz;
          if (!(r2 > rc2 && r2 <= S.RcLRF2)) continue;
        }
        int2 rg = hrange[i];
        const double3 sh = box ? image_shift(bx, hs.x - cx, hs.y - cy, hs.z - cz) : make_double3(0, 0, 0);
        if (MIXED) {
          // a zero charge adds exact zeros; water groups (3 atoms) unrolled
          const R scx = ccx + (R)sh.x, scy = ccy + (R)sh.y, scz = ccz + (R)sh.z;
          if (rg.y == 3) {
#pragma unroll
            for (int k = 0; k < 3; k++) {
              R4 a = hat[rg.x + k];
              lrf_accumulate_split((float *)mt, tt, (float)a.w, (float)(a.x - scx), (float)(a.y - scy),
                                   (float)(a.z - scz));
            }
          } else {
            for (int k = 0; k < rg.y; k++) {
              R4 a = hat[rg.x + k];
              lrf_accumulate_split((float *)mt, tt, (float)a.w, (float)(a.x - scx), (float)(a.y - scy),
                                   (float)(a.z - scz));
            }
          }
        } else {
          for (int k = 0; k < rg.y; k++) {
            R4 a = hat[rg.x + k];
            if (a.w != R(0))
              lrf_accumulate<double>(m, (double)a.w, (double)a.x - cx - sh.x, (double)a.y - cy - sh.y,
                                     (double)a.z - cz - sh.z);
          }
        }
      }
      if (MIXED) {
#pragma unroll
        for (int k = 0; k < 20; k++) mtot[k][threadIdx.x] += (double)mt[k];
#pragma unroll
        for (int k = 0; k < 4; k++) mtot[20 + k][threadIdx.x] += (double)tt[k];
      }
    }
  }
  // this block's share of the sources, added to the record (zeroed by
  // k_cgp_centers)
  if (active) {
    double *L = P.lrf + (size_t)g * LRF_STRIDE;
    if (MIXED) {
      double mm[20], t4[4];
#pragma unroll
      for (int k = 0; k < 20; k++) mm[k] = mtot[k][threadIdx.x];
#pragma unroll
      for (int k = 0; k < 4; k++) t4[k] = mtot[20 + k][threadIdx.x];
      lrf_fold(mm, t4);
#pragma unroll
      for (int k = 0; k < 20; k++)
        if (mm[k] != 0.0) atomicAdd(&L[3 + k], mm[k]);
    } else {
#pragma unroll
      for (int k = 0; k < 20; k++)
        if (m[MIXED ? 0 : k] != 0.0) atomicAdd(&L[3 + k], m[MIXED ? 0 : k]);
    }
  }
}

// -------------------------------------------- packed FP32x2 LRF gather

// lrf_accumulate_split for two target groups at once (.x and .y), on the
// packed FP32x2 pipes.  Sign conventions differ so that every update is one
// fused multiply-add: m[1..3] hold +sum f0*d (phi1 = -m[1..3]), m[10..19] and
// t[1..3] hold the phi3 sums with f2 taken positive (phi3 = -(fold of them));
// lrf_finish_x2 restores the signs.
// sel is 1 for a target inside the pair's window and 0 outside it (its
// charge q is then 0); unsel = 1 - sel.  A half outside the window may sit at
// distance 0 (a one-atom group against itself), so its r2 is replaced by 1
// before the reciprocal: every term of that half is then an exact 0.
__device__ __forceinline__ void lrf_accumulate_x2(float2 *m, float2 *t, float2 q, float2 dx, float2 dy, float2 dz,
                                                  float2 sel, float2 unsel) {
  const float2 three = make_float2(3.f, 3.f), five = make_float2(5.f, 5.f);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  const float2 r2s = __ffma2_rn(r2, sel, unsel);
  const float2 rinv = make_float2(rsqrt_ftz(r2s.x), rsqrt_ftz(r2s.y));
  const float2 ri2 = __fmul2_rn(rinv, rinv);
  const float2 f0 = __fmul2_rn(__fmul2_rn(q, rinv), ri2);          // q / r^3
  m[0] = __ffma2_rn(f0, r2, m[0]);
  m[1] = __ffma2_rn(f0, dx, m[1]); m[2] = __ffma2_rn(f0, dy, m[2]); m[3] = __ffma2_rn(f0, dz, m[3]);
  t[0] = __fadd2_rn(t[0], f0);
  const float2 f1 = __fmul2_rn(__fmul2_rn(f0, ri2), three);        // 3 q / r^5
  const float2 ax = __fmul2_rn(f1, dx), ay = __fmul2_rn(f1, dy), az = __fmul2_rn(f1, dz);
  m[4] = __ffma2_rn(ax, dx, m[4]); m[5] = __ffma2_rn(ax, dy, m[5]); m[6] = __ffma2_rn(ax, dz, m[6]);
  m[7] = __ffma2_rn(ay, dy, m[7]); m[8] = __ffma2_rn(ay, dz, m[8]); m[9] = __ffma2_rn(az, dz, m[9]);
  const float2 f2 = __fmul2_rn(f1, ri2);                            // 3 q / r^7 (the negated f2)
  const float2 w = __fmul2_rn(f2, r2);
  t[1] = __ffma2_rn(w, dx, t[1]); t[2] = __ffma2_rn(w, dy, t[2]); t[3] = __ffma2_rn(w, dz, t[3]);
  const float2 u = __fmul2_rn(f2, five);
  const float2 px = __fmul2_rn(u, dx), py = __fmul2_rn(u, dy), pz = __fmul2_rn(u, dz);
  const float2 qxx = __fmul2_rn(px, dx), qxy = __fmul2_rn(px, dy), qxz = __fmul2_rn(px, dz);
  const float2 qyy = __fmul2_rn(py, dy), qyz = __fmul2_rn(py, dz), qzz = __fmul2_rn(pz, dz);
  m[10] = __ffma2_rn(qxx, dx, m[10]); m[11] = __ffma2_rn(qxx, dy, m[11]); m[12] = __ffma2_rn(qxx, dz, m[12]);
  m[13] = __ffma2_rn(qxy, dy, m[13]); m[14] = __ffma2_rn(qxy, dz, m[14]); m[15] = __ffma2_rn(qxz, dz, m[15]);
  m[16] = __ffma2_rn(qyy, dy, m[16]); m[17] = __ffma2_rn(qyy, dz, m[17]); m[18] = __ffma2_rn(qyz, dz, m[18]);
  m[19] = __ffma2_rn(qzz, dz, m[19]);
}

// One target's packed sums (half h of every float2) as the record's 20
// components in FP64: the diagonal terms folded in, the signs restored.
__device__ __forceinline__ void lrf_finish_x2(const float2 *m, const float2 *t, int h, double *out) {
  double tt[4];
#pragma unroll
  for (int k = 0; k < 20; k++) out[k] = (double)(h ? m[k].y : m[k].x);
#pragma unroll
  for (int k = 0; k < 4; k++) tt[k] = (double)(h ? t[k].y : t[k].x);
  lrf_fold(out, tt);
#pragma unroll
  for (int k = 1; k < 4; k++) out[k] = -out[k];
#pragma unroll
  for (int k = 10; k < 20; k++) out[k] = -out[k];
}

// The mixed-precision LRF gather (nbpp/pw/wwlist_lrf, md.f90:5448, 6864,
// 8370) with two target groups per thread: targets gl and gl + LRFX_BLOCK of
// the block's chunk of 2*LRFX_BLOCK groups, each source charge applied to
// both with packed FP32x2 arithmetic (a target outside the pair's window
// takes a zero charge).  Source tiles are staged as in k_lrf_gather, atom
// positions and charges duplicated into both halves of their float2 words;
// the group-pair window test is FP64.  Each block sums its tiles in FP32 and
// adds the totals to the FP64 record with one atomic per component.
constexpr int LRFX_BLOCK = 128, LRFX_TARGETS = 2 * LRFX_BLOCK;

template <bool BOX>
__global__ void __launch_bounds__(LRFX_BLOCK, 4) k_lrf_gather_x2(DevPtrs P, int force) {
  const int s = blockIdx.y;
  if (!list_due(P, s, force)) return;
  const SysDev &S = P.sys[s];
  if (!S.use_lrf) return;
  const int tpb = P.lrf_tpb;
  const int hsplit = (S.nlrft + tpb - 1) / tpb;
  const int gchunk = blockIdx.x / max(hsplit, 1), hpart = blockIdx.x % max(hsplit, 1);
  if (hsplit == 0 || gchunk * LRFX_TARGETS >= S.ncgp) return;
  const int t0 = hpart * tpb, t1 = min(t0 + tpb, S.nlrft);
  __shared__ double4 hsw[LRF_TILE_G];
  __shared__ int2 hrange[LRF_TILE_G];
  __shared__ float4 hxy[LRF_TILE_A], hzq[LRF_TILE_A];   // {x, x, y, y}, {z, z, q, q}
  const double ox = S.origin[0], oy = S.origin[1], oz = S.origin[2];
  int gl[2];
  bool act[2], gsol[2];
  double3 xs[2], cen[2];
  float cc[2][3];
#pragma unroll
  for (int h = 0; h < 2; h++) {
    gl[h] = gchunk * LRFX_TARGETS + h * LRFX_BLOCK + threadIdx.x;
    act[h] = gl[h] < S.ncgp;
    gsol[h] = gl[h] < S.ncgp_sol;
    xs[h] = cen[h] = make_double3(0, 0, 0);
    cc[h][0] = cc[h][1] = cc[h][2] = 0.f;
    if (act[h]) {
      const int g = S.coff + gl[h];
      const int swg = P.cg_sw[g];
      act[h] = !(P.flags[swg] & F_EXCL);
      const double *L = P.lrf + (size_t)g * LRF_STRIDE;
      cen[h] = make_double3(L[0], L[1], L[2]);
      cc[h][0] = (float)(L[0] - ox); cc[h][1] = (float)(L[1] - oy); cc[h][2] = (float)(L[2] - oz);
      xs[h] = ld3(P.x, swg);
    }
  }
  // minus the two target centres (positions relative to the origin); in a
  // periodic box each source group shifts them by its image (nbpplist_box_lrf
  // md.f90:5751-5849, nbpwlist_box_lrf 7111-7245, nbwwlist_box_lrf 8601-8694)
  float2 ncx = make_float2(-cc[0][0], -cc[1][0]), ncy = make_float2(-cc[0][1], -cc[1][1]),
         ncz = make_float2(-cc[0][2], -cc[1][2]);
  const BoxD bx = box_of(P, s);
  float2 m[20], t[4];
#pragma unroll
  for (int k = 0; k < 20; k++) m[k] = make_float2(0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 4; k++) t[k] = make_float2(0.f, 0.f);
  for (int tt = t0; tt < t1; tt++) {
    const int2 tile = P.lrft[S.lrft_off + tt];
    const int nh = tile.y - tile.x;
    const int a0 = P.cg_first[S.coff + tile.x];
    const int na = P.cg_last[S.coff + tile.y - 1] - a0 + 1;
    __syncthreads();
    for (int i = threadIdx.x; i < nh; i += LRFX_BLOCK) {
      const int h = S.coff + tile.x + i;
      const int sw = P.cg_sw[h];
      const double3 p = ld3(P.x, sw);
      const double w = (P.flags[sw] & F_EXCL) ? -1.0 : (tile.x + i < S.ncgp_sol ? 1.0 : 0.0);
      hsw[i] = make_double4(p.x, p.y, p.z, w);
      hrange[i] = make_int2(P.cg_first[h] - a0, P.cg_last[h] - P.cg_first[h] + 1);
    }
    for (int i = threadIdx.x; i < na; i += LRFX_BLOCK) {
      const int at = P.cg_atoms[a0 + i];
      const double4 p = P.x[at];
      const bool qsol = (at - S.aoff) < S.nsol && P.iq[at] >= 0;
      const float x = (float)(p.x - ox), y = (float)(p.y - oy), z = (float)(p.z - oz);
      const float q = qsol ? 0.f : P.crg[at];
      hxy[i] = make_float4(x, x, y, y);
      hzq[i] = make_float4(z, z, q, q);
    }
    __syncthreads();
    if (!(act[0] || act[1])) continue;
    for (int i = 0; i < nh; i++) {
      const double4 hs = hsw[i];
      if (hs.w < 0.0) continue;
      float2 sel;
      bool any = false;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const double rc2 = (gsol[h] && hs.w > 0.0) ? S.Rcpp2 : ((gsol[h] || hs.w > 0.0) ? S.Rcpw2 : S.Rcww2);
        bool in;
        if (!S.switch_atoms && (gsol[h] || hs.w > 0.0)) {
          in = act[h] && tile.x + i != gl[h] &&
               lrf_window_any(P, S, S.coff + gl[h], gsol[h], S.coff + tile.x + i, hs.w > 0.0, rc2);
        } else {
          double dx = xs[h].x - hs.x, dy = xs[h].y - hs.y, dz = xs[h].z - hs.z;
          if (BOX) min_image(bx, dx, dy, dz);
          const double r2 = dx * dx + dy * dy + dz * dz;
          in = act[h] && tile.x + i != gl[h] && r2 > rc2 && r2 <= S.RcLRF2;
        }
        any = any || in;
        (h ? sel.y : sel.x) = in ? 1.f : 0.f;
      }
      if (!any) continue;
      if (BOX) {
        double3 c[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const double3 sh = image_shift(bx, hs.x - cen[h].x, hs.y - cen[h].y, hs.z - cen[h].z);
          c[h] = make_double3((cen[h].x - ox) + sh.x, (cen[h].y - oy) + sh.y, (cen[h].z - oz) + sh.z);
        }
        ncx = make_float2(-(float)c[0].x, -(float)c[1].x);
        ncy = make_float2(-(float)c[0].y, -(float)c[1].y);
        ncz = make_float2(-(float)c[0].z, -(float)c[1].z);
      }
      const int2 rg = hrange[i];
      const float2 unsel = make_float2(1.f - sel.x, 1.f - sel.y);
      auto atom = [&](int k) {
        const float4 a = hxy[rg.x + k], b = hzq[rg.x + k];
        const float2 q = __fmul2_rn(make_float2(b.z, b.w), sel);
        lrf_accumulate_x2(m, t, q, __fadd2_rn(make_float2(a.x, a.y), ncx), __fadd2_rn(make_float2(a.z, a.w), ncy),
                          __fadd2_rn(make_float2(b.x, b.y), ncz), sel, unsel);
      };
      if (rg.y == 3) {        // a water: its three atoms as independent chains
        atom(0);
        atom(1);
        atom(2);
      } else {
        for (int k = 0; k < rg.y; k++) atom(k);
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 2; h++) {
    if (!act[h]) continue;
    double out[20];
    lrf_finish_x2(m, t, h, out);
    double *L = P.lrf + (size_t)(S.coff + gl[h]) * LRF_STRIDE;
#pragma unroll
    for (int k = 0; k < 20; k++)
      if (out[k] != 0.0) atomicAdd(&L[3 + k], out[k]);
  }
}

// Water-water neighbour list (nbwwlist / nbwwlist_lrf, md.f90:8233, 8370),
// stored in both directions: water i lists every other water j inside the
// sphere whose O lies within Rcww of i's O, as local water indices in
// ascending order.  ww_sp[gw*ww_nch + c] counts the entries below the end of
// force-kernel chunk c (chunks of ww_chunk waters, a multiple of 32), so the
// force kernel finds each chunk's slice of the list directly; ww_mid[gw]
// counts the entries below i itself.
// Block = WL_WPB waters of one system, one warp per water at a time; the
// system's O positions are staged in shared memory WL_STAGE waters at a time
// in FP32, relative to the solvent centre (w = -1 for excluded waters), and
// scanned 64 at a time (two per lane, packed FP32x2) with a ballot per 32.
// The FP32 squared distance decides every pair farther than WL_EPS2 from the
// cut-off; the few within it are decided in FP64 from the coordinates, so the
// list is the reference's FP64 list exactly.  (|x| <= ~30 A from the centre:
// each FP32 coordinate is within 1.9e-6 A, r^2 near 100 A^2 within ~2e-4 A^2.)
constexpr int WL_BLOCK = 512, WL_WPB = 128, WL_STAGE = 2816;   // 44 KB of staged O positions
constexpr float WL_EPS2 = 4e-3f;

__global__ void __launch_bounds__(WL_BLOCK) k_list_ww(DevPtrs P, int force) {
  int s = blockIdx.y;
  if (!list_due(P, s, force)) return;
  const SysDev &S = P.sys[s];
  const int i0 = blockIdx.x * WL_WPB;
  if (i0 >= S.nwat) return;
  const int i1 = min(i0 + WL_WPB, S.nwat);
  __shared__ float4 so[WL_STAGE];
  __shared__ int scnt[WL_WPB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = WL_BLOCK / 32;
  const int obase = S.aoff + S.nsol;
  const double cx = S.pbc ? S.origin[0] : S.xw[0], cy = S.pbc ? S.origin[1] : S.xw[1],
               cz = S.pbc ? S.origin[2] : S.xw[2];
  const float rc2 = (float)S.Rcww2;
  // periodic box (nbwwlist_box, md.f90:8298): O-O distances of the nearest
  // image; FP32 edge lengths for the scan (the few pairs near the cut-off
  // are decided in FP64)
  const bool box = S.pbc != 0;
  const BoxD bx = box_of(P, s);
  const float2 bL[3] = {dup2((float)bx.L[0]), dup2((float)bx.L[1]), dup2((float)bx.L[2])};
  const float2 biL[3] = {dup2((float)bx.iL[0]), dup2((float)bx.iL[1]), dup2((float)bx.iL[2])};
  for (int t = threadIdx.x; t < WL_WPB; t += WL_BLOCK) scnt[t] = 0;
  for (int c0 = 0; c0 < S.nwat; c0 += WL_STAGE) {
    const int cn = min(WL_STAGE, S.nwat - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < cn; t += WL_BLOCK) {
      int o = obase + 3 * (c0 + t);
      double4 x = P.x[o];
      so[t] = make_float4((float)(x.x - cx), (float)(x.y - cy), (float)(x.z - cz), (P.flags[o] & F_EXCL) ? -1.f : 1.f);
    }
    __syncthreads();
    for (int iw = i0 + warp; iw < i1; iw += nwarp) {
      const int gw = S.woff + iw;
      const int oi = obase + 3 * iw;
      if (P.flags[oi] & F_EXCL) continue;
      const double3 xi = ld3(P.x, oi);
      const float2 nx = dup2(-(float)(xi.x - cx)), ny = dup2(-(float)(xi.y - cy)), nz = dup2(-(float)(xi.z - cz));
      uint16_t *out = P.ww + (size_t)gw * P.ww_cap;
      int *sp = P.ww_sp + (size_t)gw * P.ww_nch;
      int cnt = scnt[iw - i0];
      // the next end of a force-kernel chunk at or after c0 (multiples of
      // ww_chunk from ww_chunk on): the scan passes it as a multiple of 32
      int nxt = max(P.ww_chunk, (c0 + P.ww_chunk - 1) / P.ww_chunk * P.ww_chunk);
      for (int b = 0; b < cn; b += 64) {
        // lane takes j = b + lane and b + 32 + lane
        float4 a = make_float4(0.f, 0.f, 0.f, -1.f), e = a;
        const int jl0 = b + lane, jl1 = b + 32 + lane;
        if (jl0 < cn) a = so[jl0];
        if (jl1 < cn) e = so[jl1];
        float2 dx = __fadd2_rn(make_float2(a.x, e.x), nx), dy = __fadd2_rn(make_float2(a.y, e.y), ny),
               dz = __fadd2_rn(make_float2(a.z, e.z), nz);
        if (box) {
          auto wrap = [](float2 d, float2 L, float2 iL) {
            const float2 n = make_float2(rintf(d.x * iL.x), rintf(d.y * iL.y));
            return __ffma2_rn(make_float2(-n.x, -n.y), L, d);
          };
          dx = wrap(dx, bL[0], biL[0]);
          dy = wrap(dy, bL[1], biL[1]);
          dz = wrap(dz, bL[2], biL[2]);
        }
        const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        bool ok2[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int jl = h ? jl1 : jl0, jw = c0 + jl;
          const float w = h ? e.w : a.w, rr = h ? r2.y : r2.x;
          bool ok = jl < cn && jw != iw && w > 0.f;
          if (ok) {
            if (fabsf(rr - rc2) <= WL_EPS2) {
              // near the cut-off: the reference's FP64 test
              const double3 xj = ld3(P.x, obase + 3 * jw);
              double ddx = xi.x - xj.x, ddy = xi.y - xj.y, ddz = xi.z - xj.z;
              if (box) min_image(bx, ddx, ddy, ddz);
              ok = ddx * ddx + ddy * ddy + ddz * ddz <= S.Rcww2;
            } else {
              ok = rr < rc2;
            }
          }
          ok2[h] = ok;
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int base = c0 + b + 32 * h;
          if (base == nxt) {
            if (lane == 0) sp[nxt / P.ww_chunk - 1] = min(cnt, P.ww_cap);
            nxt += P.ww_chunk;
          }
          const unsigned bal = __ballot_sync(FULL, ok2[h]);
          if (ok2[h]) {
            const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
            if (pos < P.ww_cap) out[pos] = (uint16_t)(base + lane);
          }
          // the entries below water i itself: the half of its list with j > i
          // starts there
          if (lane == 0 && iw >= base && iw < base + 32)
            P.ww_mid[gw] = min(cnt + __popc(bal & ((1u << (iw - base)) - 1u)), P.ww_cap);
          cnt += __popc(bal);
        }
      }
      if (lane == 0) scnt[iw - i0] = cnt;
      __syncwarp();
    }
  }
  __syncthreads();
  for (int iw = i0 + warp; iw < i1; iw += nwarp) {
    if (lane != 0) continue;
    const int gw = S.woff + iw;
    int cnt = (P.flags[obase + 3 * iw] & F_EXCL) ? 0 : scnt[iw - i0];
    int *sp = P.ww_sp + (size_t)gw * P.ww_nch;
    if (cnt > P.ww_cap) { set_status(&P.st[s], QB_ERR_LIST_OVERFLOW); cnt = P.ww_cap; }
    P.ww_n[gw] = cnt;
    if (cnt == 0) {
      for (int c = 0; c < P.ww_nch; c++) sp[c] = 0;
      P.ww_mid[gw] = 0;
    }
    for (int c = (S.nwat - 1) / P.ww_chunk; c < P.ww_nch; c++) sp[c] = cnt;
  }
}

// exclusions and 1-4 pairs: bits for atoms within QB_NBR_RANGE of each other
// (listex/list14), else the atoms' own lists of distant partners (the
// reference scans its whole long list, md.f90:5376-5382; each atom's partners
// are the same pairs)
__device__ __forceinline__ bool long_partner(const int *off, const int *part, int i, int j) {
  for (int k = off[i]; k < off[i + 1]; k++)
    if (part[k] == j) return true;
  return false;
}

__device__ __forceinline__ bool excluded_pair(const DevPtrs &P, const SysDev &S, int i, int j) {
  // i, j global solute atoms
  int d = j - i;
  if (d <= QB_NBR_RANGE && d >= -QB_NBR_RANGE) {
    if (d > 0) return (P.lx[i] >> (d - 1)) & 1u;
    return (P.lx[j] >> (-d - 1)) & 1u;
  }
  return long_partner(P.exo, P.exq, i, j);
}

__device__ __forceinline__ bool is14(const DevPtrs &P, const SysDev &S, int i, int j) {
  int d = j - i;
  if (d <= QB_NBR_RANGE && d >= -QB_NBR_RANGE) {
    if (d > 0) return (P.l14[i] >> (d - 1)) & 1u;
    return (P.l14[j] >> (-d - 1)) & 1u;
  }
  return long_partner(P.l14o, P.l14q, i, j);
}

__device__ __forceinline__ int ljcode(const DevPtrs &P, const SysDev &S, int gi, int gj) {
  return P.ljcod[S.ljoff + P.iac[gi] * S.natyps + P.iac[gj]];
}

// all-zero pair test (md.f90:5495-5501)
__device__ __forceinline__ bool zero_pair(const DevPtrs &P, int i, int j, int lj) {
  float qq = P.crg[i] * P.crg[j];
  return qq == 0.0f && P.lja[3 * i + lj - 1] * P.lja[3 * j + lj - 1] == 0.0 &&
         P.ljb[3 * i + lj - 1] * P.ljb[3 * j + lj - 1] == 0.0;
}

// Solute-solute pair list (nbpplist, md.f90:5175): block (ig, system),
// threads over jg.  Group pairs are taken once, by the reference's parity rule.
__global__ void k_list_pp(DevPtrs P, int force) {
  int s = blockIdx.y;
  if (!list_due(P, s, force)) return;
  const SysDev &S = P.sys[s];
  int ig = blockIdx.x;
  if (ig >= S.ncgp_sol) return;
  int gi = S.coff + ig;
  int swi = P.cg_sw[gi];
  if (P.flags[swi] & F_EXCL) return;
  double3 xs = ld3(P.x, swi);
  const int lane = threadIdx.x & 31;
  // the pairs of group pair (gi, gj), written at out[0..] when out is given;
  // returns their number
  auto pairs = [&](int jg, int gj, int4 *out) {
    int n = 0;
    for (int ia = P.cg_first[gi]; ia <= P.cg_last[gi]; ia++) {
      int i = P.cg_atoms[ia];
      if (P.iq[i] >= 0) continue;
      for (int ja = P.cg_first[gj]; ja <= P.cg_last[gj]; ja++) {
        int j = P.cg_atoms[ja];
        if (ig == jg && i >= j) continue;
        if (P.iq[j] >= 0) continue;
        int lj = ljcode(P, S, i, j);
        if (zero_pair(P, i, j, lj)) continue;
        if (excluded_pair(P, S, i, j)) continue;
        if (is14(P, S, i, j)) lj = 3;
        if (out) out[n] = make_int4(i, j, lj, 0);
        n++;
      }
    }
    return n;
  };
  // rounds in which every lane of a warp takes part, so that a warp reserves
  // its pairs' slots with one atomic (a per-pair atomic on the system's
  // counter serialises the ~10^5 pairs of a large solute)
  for (int base = 0; base < S.ncgp_sol; base += blockDim.x) {
    const int jg = base + threadIdx.x;
    const int gj = S.coff + jg;
    bool inside = jg < S.ncgp_sol && !((ig > jg && ((ig + jg) & 1) == 0) || (ig < jg && ((ig + jg) & 1) == 1));
    if (inside) inside = !(P.flags[P.cg_sw[gj]] & F_EXCL);
    if (inside) {
      if (S.switch_atoms) {
        double3 xj = ld3(P.x, P.cg_sw[gj]);
        double dx = xs.x - xj.x, dy = xs.y - xj.y, dz = xs.z - xj.z;
        if (S.pbc) min_image(box_of(P, s), dx, dy, dz);   // nbpplist_box (md.f90:5349)
        inside = dx * dx + dy * dy + dz * dz <= S.Rcpp2;
      } else {
        const int reach = groups_reach(P, gi, gj, S.Rcpp2);
        double last;
        inside = reach > 0 || (reach == 0 && groups_inside_any(P, gi, gj, S.Rcpp2, &last));
      }
    }
    const int n = inside ? pairs(jg, gj, nullptr) : 0;
    // exclusive prefix of n over the warp, one reservation per warp
    int pre = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, pre, o);
      if (lane >= o) pre += t;
    }
    const int total = __shfl_sync(FULL, pre, 31);
    int first = 0;
    if (lane == 0 && total > 0) first = atomicAdd(&P.st[s].pp_n, total);
    first = __shfl_sync(FULL, first, 0);
    if (n == 0) continue;
    const int k = first + pre - n;
    if (k + n <= S.pp_cap) {
      pairs(jg, gj, P.pp + S.pp_off + k);
    } else {
      set_status(&P.st[s], QB_ERR_LIST_OVERFLOW);
    }
  }
}

// Solute-water list (nbpwlist, md.f90:6684): per solute charge group, the
// waters whose O lies within Rcpw of the group's switching atom (neither
// excluded), as local water indices in ascending order.  The pairs are the
// group's non-Q atoms with the three atoms of each listed water; pairs the
// reference drops as all-zero (md.f90:5495) contribute exact zeros here.
// One warp per solute group.
__global__ void k_list_pw(DevPtrs P, int force) {
  int s = blockIdx.y;
  if (!list_due(P, s, force)) return;
  const SysDev &S = P.sys[s];
  int ig = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (ig >= S.ncgp_sol) return;
  int gi = S.coff + ig, sg = S.csoff + ig;
  int swi = P.cg_sw[gi];
  uint16_t *out = P.pwg + (size_t)sg * P.pwg_cap;
  int cnt = 0;
  if (!(P.flags[swi] & F_EXCL)) {
    double3 xs = ld3(P.x, swi);
    for (int base = 0; base < S.nwat; base += 32) {
      int iw = base + lane;
      int o = S.aoff + S.nsol + 3 * iw;
      bool ok = false;
      if (iw < S.nwat && !(P.flags[o] & F_EXCL)) {
        double3 xo = ld3(P.x, o);
        if (S.switch_atoms) {
          double dx = xs.x - xo.x, dy = xs.y - xo.y, dz = xs.z - xo.z;
          if (S.pbc) min_image(box_of(P, s), dx, dy, dz);   // nbpwlist_box (md.f90:6801)
          ok = dx * dx + dy * dy + dz * dz <= S.Rcpw2;
        } else {
          const int reach = group_point_reach(P, gi, xo, S.Rcpw2);
          double last;
          ok = reach > 0 || (reach == 0 && group_point_inside_any(P, gi, xo, S.Rcpw2, &last));
        }
      }
      unsigned bal = __ballot_sync(FULL, ok);
      if (ok) {
        int pos = cnt + __popc(bal & ((1u << lane) - 1u));
        if (pos < P.pwg_cap) out[pos] = (uint16_t)iw;
      }
      cnt += __popc(bal);
    }
  }
  if (lane == 0) {
    if (cnt > P.pwg_cap) { set_status(&P.st[s], QB_ERR_LIST_OVERFLOW); cnt = P.pwg_cap; }
    P.pwg_n[sg] = cnt;
    int nat = 0;
    for (int a = P.cg_first[gi]; a <= P.cg_last[gi]; a++) nat += P.iq[P.cg_atoms[a]] < 0;
    if (cnt * nat) atomicAdd(&P.st[s].pw_n, 3 * cnt * nat);
  }
}

// Q-atom / solute list (nbqplist, md.f90:7875): block per system, threads
// over solute atoms of groups within Rcq of the solute centre; atoms bonded
// within 1-3 to any Q atom (in any state) belong to the Q-Q list instead.
__global__ void k_list_qp(DevPtrs P, int force) {
  int s = blockIdx.x;
  const SysDev &S = P.sys[s];
  if (S.nq == 0 || !list_due(P, s, force)) return;
  if (S.qp_once && P.st[s].lists_built) return;
  __syncthreads();
  if (threadIdx.x == 0) P.st[s].qp_n = 0;
  __syncthreads();
  // the list's centre: the solute centre, or in a periodic box the nearest
  // image of the Q switching atom (nbqplist_box, md.f90:8005-8014)
  const double3 xq = S.pbc ? ld3(P.x, S.qswitch) : make_double3(S.xp[0], S.xp[1], S.xp[2]);
  const BoxD bx = box_of(P, s);
  for (int ig = 0; ig < S.ncgp_sol; ig++) {
    int gi = S.coff + ig;
    int sw = P.cg_sw[gi];
    if (P.flags[sw] & F_EXCL) continue;
    if (S.switch_atoms) {
      double3 xs = ld3(P.x, sw);
      double dx = xs.x - xq.x, dy = xs.y - xq.y, dz = xs.z - xq.z;
      if (S.pbc) min_image(bx, dx, dy, dz);
      if (dx * dx + dy * dy + dz * dz > S.Rcq2) continue;
    } else {
      double last;
      if (!group_point_inside_any(P, gi, make_double3(S.xp[0], S.xp[1], S.xp[2]), S.Rcq2, &last)) continue;
    }
    int f = P.cg_first[gi], n = P.cg_last[gi] - f + 1;
    // whole warps per round: a warp reserves its entries with one atomic
    for (int t0 = 0; t0 < n * S.nq; t0 += blockDim.x) {
      const int t = t0 + threadIdx.x;
      bool take = t < n * S.nq;
      int i = 0, iq = 0, li = 0;
      if (take) {
        i = P.cg_atoms[f + t / S.nq];
        iq = t % S.nq;
        li = i - S.aoff;
        for (int st = 0; st < S.S && take; st++)
          for (int q = 0; q < S.nq; q++)
            if (P.qconn[S.qconn_off + ((size_t)st * S.nsol + li) * S.nq + q] <= 3) { take = false; break; }
      }
      const unsigned bal = __ballot_sync(FULL, take);
      const int lane = threadIdx.x & 31;
      int first = 0;
      if (lane == 0 && bal) first = atomicAdd(&P.st[s].qp_n, __popc(bal));
      first = __shfl_sync(FULL, first, 0);
      if (!take) continue;
      int qa = P.iqseq[S.qoff + iq];
      int lj = ljcode(P, S, i, qa);
      if (P.qconn[S.qconn_off + ((size_t)0 * S.nsol + li) * S.nq + iq] == 4) lj = 3;
      int qlj = lj == 2 ? 1 : lj;
      int k = first + __popc(bal & ((1u << lane) - 1u));
      if (k < S.qp_cap) P.qp[S.qp_off + k] = make_int4(S.qoff + iq, i, lj, qlj);
      else set_status(&P.st[s], QB_ERR_LIST_OVERFLOW);
    }
  }
}

// Q-atom / water list (nbqwlist, md.f90:8066): waters with O within Rcq of the
// solute centre.  Block per system; order of the list follows the waters.
__global__ void k_list_qw(DevPtrs P, int force) {
  int s = blockIdx.x;
  const SysDev &S = P.sys[s];
  if (S.nq == 0 || !list_due(P, s, force)) return;
  if (S.qp_once && P.st[s].lists_built) return;
  __shared__ int base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  // periodic box: the nearest image of the Q switching atom (nbqwlist_box, md.f90:8149)
  const double3 xq = S.pbc ? ld3(P.x, S.qswitch) : make_double3(S.xp[0], S.xp[1], S.xp[2]);
  const BoxD bx = box_of(P, s);
  for (int w0 = 0; w0 < S.nwat; w0 += blockDim.x) {
    int iw = w0 + threadIdx.x;
    bool ok = false;
    int o = S.aoff + S.nsol + 3 * iw;
    if (iw < S.nwat && !(P.flags[o] & F_EXCL)) {
      double3 xo = ld3(P.x, o);
      double dx = xo.x - xq.x, dy = xo.y - xq.y, dz = xo.z - xq.z;
      if (S.pbc) min_image(bx, dx, dy, dz);
      ok = dx * dx + dy * dy + dz * dz <= S.Rcq2;
    }
    // block-wide ordered compaction
    __shared__ int wcount[32];
    unsigned bal = __ballot_sync(FULL, ok);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) wcount[wid] = __popc(bal);
    __syncthreads();
    int off = base;
    for (int w = 0; w < wid; w++) off += wcount[w];
    if (ok) {
      int k = off + __popc(bal & ((1u << lane) - 1u));
      if (k < S.qw_cap) P.qw[S.qw_off + k] = o;
      else set_status(&P.st[s], QB_ERR_LIST_OVERFLOW);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) tot += wcount[w];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) P.st[s].qw_n = base < S.qw_cap ? base : S.qw_cap;
}

// Per-run counters (SHAKE iterations) back to zero.
__global__ void k_reset_counters(DevPtrs P) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nsys) return;
  P.st[s].shake_its = 0;
  P.st[s].shake_its_max = 0;
}
__global__ void k_lists_begin(DevPtrs P, int force) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nsys || !list_due(P, s, force)) return;
  P.st[s].pp_n = 0;
  P.st[s].pw_n = 0;
}

__global__ void k_lists_end(DevPtrs P, int force) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= P.nsys || !list_due(P, s, force)) return;
  SysState &st = P.st[s];
  const SysDev &S = P.sys[s];
  if (st.pp_n > S.pp_cap) st.pp_n = S.pp_cap;
  if (st.qp_n > S.qp_cap) st.qp_n = S.qp_cap;
  st.lists_built = 1;
}

// ------------------------------------------------------------- nonbonded

// Per-water position records of the water-water kernel, 16-byte words.
// FP64 (5 words, 80 bytes): O,H1,H2 x,y,z as doubles and one pad double.
// Mixed (3 words, 48 bytes): the O position as an unevaluated float sum
// hi + lo (hi = float(x), lo = float(x - hi)) and the two H positions relative
// to their O, rounded to float: {hO.xyz, lO.x}, {lO.yz, rH1.x, rH2.x},
// {rH1.y, rH2.y, rH1.z, rH2.z} -- each component's two H offsets side by
// side, one packed FP32x2 operand.  An atom-pair vector is then
// ((hOj - hOi) + (lOj - lOi)) + rHj - rHi, which carries ~1e-7 relative error
// like an FP64 difference rounded to FP32.  Both strides (3 and 5 words) put
// 8 consecutive waters on 8 distinct 16-byte bank groups.
template <bool MIXED> struct WatRec { static constexpr int words = MIXED ? 3 : 5; };
constexpr int WREC_MAX = 5;
// threads, most waters per block (a batch of few systems takes fewer per
// block, so that its blocks still fill the SMs)
constexpr int WW_BLOCK = 512, WW_WPB = 256;   // threads, most waters per block
constexpr int WW_STAGE_BYTES = 112 * 1024;    // staged records per block: two blocks per SM

// watpol (md.f90:15122), per water: the angle between the water dipole and
// the radius vector from the restraint centre, and the polarisation shell the
// O lies in (-1: none, or excluded).
__device__ __forceinline__ void watpol_angle(const DevPtrs &P, const SysDev &S, int gw, bool excl, double4 xO,
                                             double4 x1, double4 x2) {
  int shell = -1;
  double theta = 0.0;
  if (!excl) {
    double rmu[3] = {x1.x + x2.x - 2. * xO.x, x1.y + x2.y - 2. * xO.y, x1.z + x2.z - 2. * xO.z};
    double rm = sqrt(rmu[0] * rmu[0] + rmu[1] * rmu[1] + rmu[2] * rmu[2]);
    for (int k = 0; k < 3; k++) rmu[k] /= rm;
    double rcu[3] = {xO.x - S.xw[0], xO.y - S.xw[1], xO.z - S.xw[2]};
    double rc = sqrt(rcu[0] * rcu[0] + rcu[1] * rcu[1] + rcu[2] * rcu[2]);
    for (int k = 0; k < 3; k++) rcu[k] /= rc;
    double scp = rmu[0] * rcu[0] + rmu[1] * rcu[1] + rmu[2] * rcu[2];
    if (scp > 1.0) scp = 1.0;
    if (scp < -1.0) scp = -1.0;
    theta = acos(scp);
    const int ns = S.nshell;
    float inner = S.ws_rout[ns - 1] - S.ws_dr[ns - 1];
    if (rc > (double)inner) {
      int is;
      for (is = ns - 1; is >= 1; is--)
        if (rc <= (double)S.ws_rout[is]) break;
      shell = is;
    }
  }
  P.wtheta[gw] = theta;
  P.wshell[gw] = (int8_t)shell;
}


// One SPC/TIP3P molecule pair (md.f90:11823-11950, nonbond_ww_spc): the 9
// Coulomb terms and the O-O Lennard-Jones term, gradient of molecule i added
// to f[9].  HLJ adds the O-H and H-H Lennard-Jones terms of nonbon2_ww
// (md.f90:10099) and nonbond_3atomsolvent (12317); lj = {A, B} of O-O, O-H, H-H.
template <bool HLJ>
__device__ __forceinline__ void ww_pair_f64(const double *xi, const double *xj, double qoo, double qoh, double qhh,
                                            const double *lj, double *f, double &el, double &vdw) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      double dx = xj[3 * b] - xi[3 * a], dy = xj[3 * b + 1] - xi[3 * a + 1], dz = xj[3 * b + 2] - xi[3 * a + 2];
      double rinv = rsqrt(dx * dx + dy * dy + dz * dz);
      double r2 = rinv * rinv;
      double qq = (a == 0 && b == 0) ? qoo : ((a == 0 || b == 0) ? qoh : qhh);
      double Vel = qq * rinv, dv;
      if ((a == 0 && b == 0) || HLJ) {
        const int t = (a == 0 && b == 0) ? 0 : ((a == 0 || b == 0) ? 2 : 4);
        double r6 = r2 * r2 * r2;
        double Va = lj[t] * r6 * r6, Vb = lj[t + 1] * r6;
        vdw += Va - Vb;
        dv = r2 * (-Vel - 12. * Va + 6. * Vb);
      } else {
        dv = r2 * (-Vel);
      }
      el += Vel;
      f[3 * a + 0] -= dv * dx;
      f[3 * a + 1] -= dv * dy;
      f[3 * a + 2] -= dv * dz;
    }
}

// Mixed precision: i = {hO[3], lO[3], rH1[3], rH2[3]}, j likewise.
// sh: the molecule pair's periodic image shift as hi + lo floats ({hi[3],
// lo[3]}), or nullptr.
template <bool HLJ>
__device__ __forceinline__ void ww_pair_f32(const float *i, const float *j, float qoo, float qoh, float qhh,
                                            const float *lj, float *f, float &el, float &vdw,
                                            const float *sh = nullptr) {
  float dOO[3], t[2][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    dOO[c] = sh ? ((j[c] - i[c]) - sh[c]) + ((j[3 + c] - i[3 + c]) - sh[3 + c]) : (j[c] - i[c]) + (j[3 + c] - i[3 + c]);
    t[0][c] = dOO[c] + j[6 + c];
    t[1][c] = dOO[c] + j[9 + c];
  }
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      float d[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float v = b == 0 ? dOO[c] : t[b - 1][c];
        d[c] = a == 0 ? v : v - i[3 + 3 * a + c];
      }
      float rinv = rsqrt_ftz(fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2])));
      float r2 = rinv * rinv;
      float qq = (a == 0 && b == 0) ? qoo : ((a == 0 || b == 0) ? qoh : qhh);
      float Vel = qq * rinv, dv;
      if ((a == 0 && b == 0) || HLJ) {
        const int t = (a == 0 && b == 0) ? 0 : ((a == 0 || b == 0) ? 2 : 4);
        float r6 = r2 * r2 * r2;
        float Va = lj[t] * r6 * r6, Vb = lj[t + 1] * r6;
        vdw += Va - Vb;
        dv = r2 * (-Vel - 12.f * Va + 6.f * Vb);
      } else {
        dv = -r2 * Vel;
      }
      el += Vel;
#pragma unroll
      for (int c = 0; c < 3; c++) f[3 * a + c] = fmaf(-dv, d[c], f[3 * a + c]);
    }
}

// Mixed record -> {hO[3], lO[3], rH1[3], rH2[3]}.
__device__ __forceinline__ void unpack_mixed(const float4 *r, float *v) {
  float4 w0 = r[0], w1 = r[1], w2 = r[2];
  v[0] = w0.x; v[1] = w0.y; v[2] = w0.z; v[3] = w0.w; v[4] = w1.x; v[5] = w1.y;
  v[6] = w1.z; v[7] = w2.x; v[8] = w2.z; v[9] = w1.w; v[10] = w2.y; v[11] = w2.w;
}

// nonbond_ww_spc (md.f90:11823) over the water-water list.  Block = 512
// threads on wpb (<= WW_WPB) consecutive waters of one system (blockIdx.y).  The
// system's water records are staged in shared memory in chunks of ww_chunk
// waters; for each chunk every half-warp takes one water i and its 16 lanes
// walk i's list slice for that chunk (the next entry prefetched), so
// neighbour records come from shared memory.  Gradients of i are reduced over
// the half-warp and added once per chunk; each unordered pair is evaluated
// from both sides, energies halved.  Mixed precision: pair terms in FP32
// (MUFU rsqrt), each lane's energy over one water's list slice summed in FP32 and accumulated in
// FP64, gradients reduced in FP32.
// EONCE (FP64 only): the energies alone, each unordered pair once (the list
// entries above ww_mid, j > i) and not halved; the mixed engine's recording
// steps take these beside the packed kernel's forces.
template <bool MIXED, bool HLJ, bool EONCE = false>
__global__ void __launch_bounds__(WW_BLOCK, MIXED ? 2 : 1) k_nb_ww(DevPtrs P, int wpb) {
  static_assert(!(MIXED && EONCE), "energies-only form is FP64");
  extern __shared__ float4 wsm[];
  __shared__ int2 srange[WW_WPB];          // list slice of each of the block's waters in this chunk
  constexpr int W = WatRec<MIXED>::words;
  // the block's (system, first water) from the batch's tile list: no empty
  // blocks for the systems with fewer waters
  const int2 tile = P.ww_tiles[blockIdx.x];
  const int s = tile.x;
  const SysDev &S = P.sys[s];
  const int i0 = tile.y;
  const int i1 = min(i0 + wpb, S.nwat);
  const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const float4 *rec = (MIXED ? P.wrec32 : P.wrec) + (size_t)S.woff * W;
  const int CW = P.ww_chunk;
  const int nch = (S.nwat + CW - 1) / CW;
  const float qo = S.crg_ow, qh = S.crg_hw;
  // periodic box (nonbond_ww_spc_box, md.f90:12078-12100): molecule j at the
  // image of its O nearest i's O
  const bool box = S.pbc != 0;
  const BoxD bx = box_of(P, s);
  double el = 0, vdw = 0;
  for (int c = 0; c < nch; c++) {
    const int c0 = c * CW, cn = min(CW, S.nwat - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < cn * W; t += WW_BLOCK) wsm[t] = rec[(size_t)c0 * W + t];
    for (int t = threadIdx.x; t < i1 - i0; t += WW_BLOCK) {
      const int *sp = P.ww_sp + (size_t)(S.woff + i0 + t) * P.ww_nch;
      int lo = c == 0 ? 0 : sp[c - 1];
      if (EONCE) lo = max(lo, P.ww_mid[S.woff + i0 + t]);
      srange[t] = make_int2(lo, sp[c]);
    }
    __syncthreads();
    // first list entry of the half-warp's next water, fetched one water ahead
    int jn_next = c0;
    {
      const int iw = i0 + hw;
      if (iw < i1) {
        const int2 r = srange[iw - i0];
        if (r.x + hl < r.y) jn_next = P.ww[(size_t)(S.woff + iw) * P.ww_cap + r.x + hl];
      }
    }
    for (int iw = i0 + hw; iw < i1; iw += WW_BLOCK / 16) {
      const int gw = S.woff + iw;
      const int kb = srange[iw - i0].x, ke = srange[iw - i0].y;
      int jn = jn_next;
      {
        const int iw2 = iw + WW_BLOCK / 16;
        jn_next = c0;
        if (iw2 < i1) {
          const int2 r = srange[iw2 - i0];
          if (r.x + hl < r.y) jn_next = P.ww[(size_t)(S.woff + iw2) * P.ww_cap + r.x + hl];
        }
      }
      if (kb >= ke) continue;
      const uint16_t *nb = P.ww + (size_t)gw * P.ww_cap;
      const float4 *ri = (iw >= c0 && iw < c0 + cn) ? wsm + (iw - c0) * W : rec + (size_t)iw * W;
      const int oi = S.aoff + S.nsol + 3 * iw;
      double fd[9];
      int k = kb + hl;
      if (MIXED) {
        float xi[12];
        unpack_mixed(ri, xi);
        const float qoo = qo * qo, qoh = qo * qh, qhh = qh * qh;
        const float ljf[6] = {(float)S.A_OO, (float)S.B_OO, (float)S.A_OH, (float)S.B_OH, (float)S.A_HH, (float)S.B_HH};
        float f[9];
#pragma unroll
        for (int q = 0; q < 9; q++) f[q] = 0.f;
        float e_el = 0.f, e_vdw = 0.f;
        int jn2 = k + 16 < ke ? (int)nb[k + 16] : c0;     // two entries in flight
        for (; k < ke; k += 16) {
          const int j = jn;
          jn = jn2;
          if (k + 32 < ke) jn2 = nb[k + 32];
          float xj[12];
          unpack_mixed(wsm + (j - c0) * W, xj);
          if (box) {
            float sh[6];
#pragma unroll
            for (int q = 0; q < 3; q++) {
              const double d = ((double)xj[q] + (double)xj[3 + q]) - ((double)xi[q] + (double)xi[3 + q]);
              const double t = bx.L[q] * round(d * bx.iL[q]);
              sh[q] = (float)t;
              sh[3 + q] = (float)(t - (double)sh[q]);
            }
            ww_pair_f32<HLJ>(xi, xj, qoo, qoh, qhh, ljf, f, e_el, e_vdw, sh);
          } else {
            ww_pair_f32<HLJ>(xi, xj, qoo, qoh, qhh, ljf, f, e_el, e_vdw);
          }
        }
        el += (double)e_el;
        vdw += (double)e_vdw;
#pragma unroll
        for (int q = 0; q < 9; q++) {
          float t = f[q];
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) t += __shfl_xor_sync(hmask, t, o);
          fd[q] = (double)t;
        }
      } else {
        const double2 *rd = reinterpret_cast<const double2 *>(ri);
        double2 d0 = rd[0], d1 = rd[1], d2 = rd[2], d3 = rd[3], d4 = rd[4];
        const double xi[9] = {d0.x, d0.y, d1.x, d1.y, d2.x, d2.y, d3.x, d3.y, d4.x};
        const double qoo = (double)(qo * qo), qoh = (double)(qo * qh), qhh = (double)(qh * qh);
        const double ljd[6] = {S.A_OO, S.B_OO, S.A_OH, S.B_OH, S.A_HH, S.B_HH};
#pragma unroll
        for (int q = 0; q < 9; q++) fd[q] = 0.0;
        for (; k < ke; k += 16) {
          const int j = jn;
          if (k + 16 < ke) jn = nb[k + 16];
          const double2 *rj = reinterpret_cast<const double2 *>(wsm + (j - c0) * W);
          double2 v0 = rj[0], v1 = rj[1], v2 = rj[2], v3 = rj[3], v4 = rj[4];
          double xj[9] = {v0.x, v0.y, v1.x, v1.y, v2.x, v2.y, v3.x, v3.y, v4.x};
          if (box) {
            const double3 t = image_shift(bx, xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]);
#pragma unroll
            for (int a = 0; a < 3; a++) { xj[3 * a] -= t.x; xj[3 * a + 1] -= t.y; xj[3 * a + 2] -= t.z; }
          }
          ww_pair_f64<HLJ>(xi, xj, qoo, qoh, qhh, ljd, fd, el, vdw);
        }
        if (!EONCE) {
#pragma unroll
          for (int q = 0; q < 9; q++) {
#pragma unroll
            for (int o = 8; o > 0; o >>= 1) fd[q] += __shfl_xor_sync(hmask, fd[q], o);
          }
        }
      }
      // fire-and-forget adds: the half-warp does not wait for the gradient
      if (!EONCE && hl == 0) {
#pragma unroll
        for (int a = 0; a < 3; a++) atomic_add3(P.d, oi + a, fd[3 * a], fd[3 * a + 1], fd[3 * a + 2]);
      }
    }
  }
  warp_add(&P.E[s * QB_NE + QB_E_WW_EL], EONCE ? el : 0.5 * el);
  warp_add(&P.E[s * QB_NE + QB_E_WW_VDW], EONCE ? vdw : 0.5 * vdw);
}

// ----------------------------------------------- packed FP32x2 water-water

// Operands of water i on the packed path: O as hi + lo, the H offsets negated
// in both orders ({-rH1, -rH2} and {-rH2, -rH1}, per component).
struct WwI2 {
  float hO[3], lO[3];
  float2 nrH[3], nrHs[3];
};

// Gradient of water i from molecule pair (i, j) of nonbond_ww_spc
// (md.f90:11823-11950), forces only, on Blackwell's packed FP32x2 pipes
// (FADD2/FMUL2/FFMA2: two lanes of FP32 work per issued instruction).  The
// eight H-involving Coulomb pairs are four packed pairs:
//   t  = O_i -> {H1_j, H2_j}      (into gO, both halves O_i's)
//   s  = {H1_i, H2_i} -> O_j      (into gH = {H1_i, H2_i})
//   hd = {H1_i, H2_i} -> {H1_j, H2_j}  (into gH)
//   hx = {H2_i, H1_i} -> {H1_j, H2_j}  (into gHs = {H2_i, H1_i})
// plus the O-O Lennard-Jones + Coulomb pair (into gO.x).  Each gradient term
// is w * (x_j - x_i) with w = q q / r^3 (Coulomb) and r^-2 (q q / r + 12 A /
// r^12 - 6 B / r^6) for O-O: -dv of the reference loop.
// BOX: the periodic box's edge lengths as hi + lo floats (Lh, Ll) and their
// inverses iL: the O-O vector moves to its nearest image (nonbond_ww_spc_box,
// md.f90:12078-12100; the FP32 nint agrees with the FP64 one away from half an
// edge, far beyond the cut-off).
template <bool BOX>
__device__ __forceinline__ void ww_force_x2(const WwI2 &I, const float4 j0, const float4 j1, const float4 j2,
                                            float2 qoh2, float2 qhh2, float qoo, float A, float B, float2 *gO,
                                            float2 *gH, float2 *gHs, const float *Lh = nullptr,
                                            const float *Ll = nullptr, const float *iL = nullptr) {
  float d[3] = {(j0.x - I.hO[0]) + (j0.w - I.lO[0]), (j0.y - I.hO[1]) + (j1.x - I.lO[1]),
                (j0.z - I.hO[2]) + (j1.y - I.lO[2])};
  if (BOX) {
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float n = rintf(d[c] * iL[c]);
      d[c] = fmaf(-n, Ll[c], fmaf(-n, Lh[c], d[c]));
    }
  }
  const float2 rHj[3] = {make_float2(j1.z, j1.w), make_float2(j2.x, j2.y), make_float2(j2.z, j2.w)};
  float2 t[3], sv[3], hd[3], hx[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 u = dup2(d[c]);
    t[c] = __fadd2_rn(u, rHj[c]);
    sv[c] = __fadd2_rn(u, I.nrH[c]);
    hd[c] = __fadd2_rn(t[c], I.nrH[c]);
    hx[c] = __fadd2_rn(t[c], I.nrHs[c]);
  }
  auto r2of = [](const float2 *v) { return __ffma2_rn(v[0], v[0], __ffma2_rn(v[1], v[1], __fmul2_rn(v[2], v[2]))); };
  auto wof = [](float2 r2, float2 qq) {
    const float2 ri = make_float2(rsqrt_ftz(r2.x), rsqrt_ftz(r2.y));
    return __fmul2_rn(__fmul2_rn(qq, ri), __fmul2_rn(ri, ri));
  };
  const float2 wt = wof(r2of(t), qoh2), ws = wof(r2of(sv), qoh2);
  const float2 wd = wof(r2of(hd), qhh2), wx = wof(r2of(hx), qhh2);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    gO[c] = __ffma2_rn(wt, t[c], gO[c]);
    gH[c] = __ffma2_rn(wd, hd[c], __ffma2_rn(ws, sv[c], gH[c]));
    gHs[c] = __ffma2_rn(wx, hx[c], gHs[c]);
  }
  const float r2 = fmaf(d[0], d[0], fmaf(d[1], d[1], d[2] * d[2]));
  const float ri = rsqrt_ftz(r2), r2i = ri * ri, r6 = r2i * r2i * r2i;
  const float Va = A * r6 * r6, Vb = B * r6;
  const float w = r2i * fmaf(-6.f, Vb, fmaf(12.f, Va, qoo * ri));
#pragma unroll
  for (int c = 0; c < 3; c++) gO[c].x = fmaf(w, d[c], gO[c].x);
}

// nonbond_ww_spc (md.f90:11823) forces of the mixed-precision engine on steps
// that record no energies: the list walk of k_nb_ww (half a warp per water,
// the system's records staged in shared memory chunk by chunk) with the pair
// terms of ww_force_x2.  Energies are left to the steps that record them,
// which evaluate the water-water pairs in FP64 (k_nb_ww<false>).  SPC water
// only (no hydrogen Lennard-Jones).
// 256 threads, two blocks per SM: one block's staging of records overlaps
// the other's pair work (the registers of the packed path allow 16 warps per
// SM).  A three-block form (80 registers, staging chunks of up to 74 KB) ran
// the kernel 13% slower alone, and the step no faster.
constexpr int WWX_BLOCK = 256;
template <bool BOX>
__global__ void __launch_bounds__(WWX_BLOCK, 2) k_nb_ww_x2(DevPtrs P, int wpb) {
  extern __shared__ float4 wsm[];
  __shared__ int2 srange[WW_WPB];
  constexpr int W = WatRec<true>::words;
  const int2 tile = P.ww_tiles[blockIdx.x];
  const int s = tile.x;
  const SysDev &S = P.sys[s];
  const int i0 = tile.y;
  const int i1 = min(i0 + wpb, S.nwat);
  const int hw = threadIdx.x >> 4, hl = threadIdx.x & 15;
  const unsigned hmask = (threadIdx.x & 16) ? 0xffff0000u : 0x0000ffffu;
  const float4 *rec = P.wrec32 + (size_t)S.woff * W;
  const int CW = P.ww_chunk;
  const int nch = (S.nwat + CW - 1) / CW;
  const float qo = S.crg_ow, qh = S.crg_hw;
  const float qoo = qo * qo;
  const float2 qoh2 = dup2(qo * qh), qhh2 = dup2(qh * qh);
  const float A = (float)S.A_OO, B = (float)S.B_OO;
  float Lh[3], Ll[3], iL[3];
  if (BOX) {
    const BoxD bx = box_of(P, s);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      Lh[q] = (float)bx.L[q];
      Ll[q] = (float)(bx.L[q] - (double)Lh[q]);
      iL[q] = (float)bx.iL[q];
    }
  }
  for (int c = 0; c < nch; c++) {
    const int c0 = c * CW, cn = min(CW, S.nwat - c0);
    __syncthreads();
    for (int t = threadIdx.x; t < cn * W; t += WWX_BLOCK) wsm[t] = rec[(size_t)c0 * W + t];
    for (int t = threadIdx.x; t < i1 - i0; t += WWX_BLOCK) {
      const int *sp = P.ww_sp + (size_t)(S.woff + i0 + t) * P.ww_nch;
      srange[t] = make_int2(c == 0 ? 0 : sp[c - 1], sp[c]);
    }
    __syncthreads();
    // the first group of list entries of the half-warp's next water, loaded
    // one water ahead
    int jfirst[4];
    auto first_group = [&](int iw2, int *out) {
#pragma unroll
      for (int u = 0; u < 4; u++) out[u] = -1;
      if (iw2 >= i1) return;
      const int2 r = srange[iw2 - i0];
      const uint16_t *nb2 = P.ww + (size_t)(S.woff + iw2) * P.ww_cap;
#pragma unroll
      for (int u = 0; u < 4; u++)
        if (r.x + hl + 16 * u < r.y) out[u] = nb2[r.x + hl + 16 * u];
    };
    first_group(i0 + hw, jfirst);
    for (int iw = i0 + hw; iw < i1; iw += WWX_BLOCK / 16) {
      const int gw = S.woff + iw;
      const int kb = srange[iw - i0].x, ke = srange[iw - i0].y;
      int jg[4];
#pragma unroll
      for (int u = 0; u < 4; u++) jg[u] = jfirst[u];
      first_group(iw + WWX_BLOCK / 16, jfirst);
      if (kb >= ke) continue;
      const uint16_t *nb = P.ww + (size_t)gw * P.ww_cap;
      const float4 *ri = (iw >= c0 && iw < c0 + cn) ? wsm + (iw - c0) * W : rec + (size_t)iw * W;
      WwI2 I;
      {
        const float4 a = ri[0], b = ri[1], e = ri[2];
        I.hO[0] = a.x; I.hO[1] = a.y; I.hO[2] = a.z;
        I.lO[0] = a.w; I.lO[1] = b.x; I.lO[2] = b.y;
        I.nrH[0] = make_float2(-b.z, -b.w); I.nrH[1] = make_float2(-e.x, -e.y); I.nrH[2] = make_float2(-e.z, -e.w);
#pragma unroll
        for (int q = 0; q < 3; q++) I.nrHs[q] = make_float2(I.nrH[q].y, I.nrH[q].x);
      }
      float2 gO[3], gH[3], gHs[3];
#pragma unroll
      for (int q = 0; q < 3; q++) gO[q] = gH[q] = gHs[q] = make_float2(0.f, 0.f);
      // the lane's list entries in groups of four, loaded together, the next
      // group's loads issued before the current group's pairs
      int k = kb + hl;
      for (; k < ke; k += 64) {
        int jn[4];
#pragma unroll
        for (int u = 0; u < 4; u++) jn[u] = k + 64 + 16 * u < ke ? (int)nb[k + 64 + 16 * u] : -1;
#pragma unroll
        for (int u = 0; u < 4; u++) {
          if (jg[u] < 0) break;
          const float4 *rj = wsm + (jg[u] - c0) * W;
          ww_force_x2<BOX>(I, rj[0], rj[1], rj[2], qoh2, qhh2, qoo, A, B, gO, gH, gHs, Lh, Ll, iL);
        }
#pragma unroll
        for (int u = 0; u < 4; u++) jg[u] = jn[u];
      }
      // per atom of water i: O, H1, H2 (x, y, z each), reduced over the half-warp
      float g[9];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        g[q] = gO[q].x + gO[q].y;
        g[3 + q] = gH[q].x + gHs[q].y;
        g[6 + q] = gH[q].y + gHs[q].x;
      }
#pragma unroll
      for (int q = 0; q < 9; q++) {
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) g[q] += __shfl_xor_sync(hmask, g[q], o);
      }
      if (hl == 0) {
        const int oi = S.aoff + S.nsol + 3 * iw;
#pragma unroll
        for (int a = 0; a < 3; a++)
          atomic_add3(P.d, oi + a, (double)g[3 * a], (double)g[3 * a + 1], (double)g[3 * a + 2]);
      }
    }
  }
}

// nonbond_pp (md.f90:10387): one thread per pair.
__device__ __forceinline__ void nb_pp_body(DevPtrs &P, int bx, int s, int gx) {
  const SysDev &S = P.sys[s];
  int n = P.st[s].pp_n;
  const int4 *L = P.pp + S.pp_off;
  double el = 0, vdw = 0;
  const int lane = threadIdx.x & 31;
  for (int k0 = bx * blockDim.x; k0 < n; k0 += gx * blockDim.x) {
    int k = k0 + threadIdx.x;
    // the list holds each atom i's pairs of a group pair consecutively: the
    // lanes with the same i sum their share of i's gradient over the warp and
    // the first of them adds it with one atomic per component
    double gi[3] = {0.0, 0.0, 0.0};
    int i = -1 - lane;
    if (k < n) {
      int4 p = L[k];
      i = p.x;
      int j = p.y, lj = p.z;
      double3 xi = ld3(P.x, i), xj = ld3(P.x, j);
      double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
      if (S.pbc) {
        // nonbond_pp_box (md.f90:10508-10519): the image of the charge-group
        // pair, from the two groups' switching atoms
        const double3 a = ld3(P.x, switch_of(P, i)), b = ld3(P.x, switch_of(P, j));
        const double3 t = image_shift(box_of(P, s), b.x - a.x, b.y - a.y, b.z - a.z);
        dx -= t.x; dy -= t.y; dz -= t.z;
      }
      double r = rsqrt(dx * dx + dy * dy + dz * dz);
      double r2 = r * r, r6 = r2 * r2 * r2;
      float qq = P.crg[i] * P.crg[j];
      double Vel = (double)qq * r;
      if (lj == 3) Vel = Vel * S.el14;
      double Va, Vb;
      if (S.arith) {
        double A, B;
        lj_pair(1, P.lja[3 * i + lj - 1], P.lja[3 * j + lj - 1], P.ljb[3 * i + lj - 1], P.ljb[3 * j + lj - 1], A, B);
        Va = A * r6 * r6;
        Vb = B * r6;
      } else {
        Va = r6 * r6 * P.lja[3 * i + lj - 1] * P.lja[3 * j + lj - 1];
        Vb = r6 * P.ljb[3 * i + lj - 1] * P.ljb[3 * j + lj - 1];
      }
      double dv = r2 * (-Vel - 12. * Va + 6. * Vb);
      gi[0] = -dv * dx; gi[1] = -dv * dy; gi[2] = -dv * dz;
      atomic_add3(P.d, j, dv * dx, dv * dy, dv * dz);
      el += Vel;
      vdw += Va - Vb;
    }
    // runs of equal i in consecutive lanes: a segmented sum towards each
    // run's first lane (end: the next run's first lane)
    const int prev = __shfl_up_sync(FULL, i, 1);
    const bool head = lane == 0 || prev != i;
    const unsigned heads = __ballot_sync(FULL, head);
    const unsigned later = lane == 31 ? 0u : heads & ~((2u << lane) - 1u);
    const int end = later ? __ffs(later) - 1 : 32;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const bool take = lane + o < end;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double t = __shfl_down_sync(FULL, gi[c], o);
        if (take) gi[c] += t;
      }
    }
    if (i >= 0 && head) atomic_add3(P.d, i, gi[0], gi[1], gi[2]);
  }
  warp_add(&P.E[s * QB_NE + QB_E_PP_EL], el);
  warp_add(&P.E[s * QB_NE + QB_E_PP_VDW], vdw);
}

// nonbond_pw (md.f90:10631) over the group list: one thread per (listed
// water, solute charge group); grid (water chunks, solute groups, systems).
// The group's non-Q atoms and their parameters for the water O and H sites
// (charge products in single precision, as crg(i)*crg(j); LJ products) are
// static tables read as broadcasts.  Each thread adds its water's 9 gradient
// components with atomics once; each solute atom's gradient is reduced over
// the warp and added with one atomic per warp.
constexpr int PW_BLOCK = 128, PW_MAXA = 128;   // group atoms staged in shared memory

// F32: the mixed engine's steps that record no energies take the forces
// alone in FP32 (differences of the FP64 positions rounded to FP32, MUFU
// reciprocal square root), as its water-water kernel does; energy-recording
// steps run the FP64 form.
template <bool F32>
__global__ void __launch_bounds__(PW_BLOCK) k_nb_pw(DevPtrs P) {
  const int2 sgi = P.pw_groups[blockIdx.x];   // (system, solute group)
  const int s = sgi.x;
  const SysDev &S = P.sys[s];
  const int ig = sgi.y;
  const int sg = S.csoff + ig;
  const int n = P.pwg_n[sg];
  const int k0 = blockIdx.y * PW_BLOCK;
  if (k0 >= n) return;
  const int k = k0 + threadIdx.x;
  const bool act = k < n;
  const int lane = threadIdx.x & 31;
  const int ow = S.aoff + S.nsol;
  const int o = ow + 3 * (act ? (int)P.pwg[(size_t)sg * P.pwg_cap + k] : 0);
  double3 xw[3] = {ld3(P.x, o), ld3(P.x, o + 1), ld3(P.x, o + 2)};
  if (S.pbc) {
    // nonbond_pw_box (md.f90:10693-10699): the water at the image of its O
    // nearest the group's switching atom
    const double3 a = ld3(P.x, P.cg_sw[S.coff + ig]);
    const double3 t = image_shift(box_of(P, s), xw[0].x - a.x, xw[0].y - a.y, xw[0].z - a.z);
#pragma unroll
    for (int b = 0; b < 3; b++) { xw[b].x -= t.x; xw[b].y -= t.y; xw[b].z -= t.z; }
  }
  // the group's atoms, parameters and positions staged once per block
  __shared__ PwAtom sa[PW_MAXA];
  __shared__ double4 sx[PW_MAXA];
  const int ta = P.pwg_off[sg], na = min(P.pwg_off[sg + 1] - ta, PW_MAXA);
  if (threadIdx.x < na) {
    const PwAtom A = P.pwa[ta + threadIdx.x];
    sa[threadIdx.x] = A;
    sx[threadIdx.x] = P.x[A.atom];
  }
  __syncthreads();
  double fw[9];
  float fw32[9];
#pragma unroll
  for (int c = 0; c < 9; c++) { fw[c] = 0.0; fw32[c] = 0.f; }
  double el = 0, vdw = 0;
  const int t1 = P.pwg_off[sg + 1];
  for (int t = ta; t < t1; t++) {
    const PwAtom A = t - ta < PW_MAXA ? sa[t - ta] : P.pwa[t];
    const double4 x4 = t - ta < PW_MAXA ? sx[t - ta] : P.x[A.atom];
    const double3 xi = make_double3(x4.x, x4.y, x4.z);
    double fi[3] = {0.0, 0.0, 0.0};
    if (F32) {
      // forces alone: the group atom's FP32 terms summed over the warp in FP32
      float gi[3] = {0.f, 0.f, 0.f};
#pragma unroll
      for (int b = 0; b < 3; b++) {
        if (!act) break;
        const float dx = (float)(xw[b].x - xi.x), dy = (float)(xw[b].y - xi.y), dz = (float)(xw[b].z - xi.z);
        const float r = rsqrt_ftz(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        const float r2 = r * r, r6 = r2 * r2 * r2;
        const float Vel = (b == 0 ? A.q.x : A.q.y) * r;
        const float Va = (float)(b == 0 ? A.lj.x : A.lj.z) * r6 * r6, Vb = (float)(b == 0 ? A.lj.y : A.lj.w) * r6;
        const float dv = r2 * (-Vel - 12.f * Va + 6.f * Vb);
        gi[0] = fmaf(-dv, dx, gi[0]); gi[1] = fmaf(-dv, dy, gi[1]); gi[2] = fmaf(-dv, dz, gi[2]);
        fw32[3 * b] = fmaf(dv, dx, fw32[3 * b]); fw32[3 * b + 1] = fmaf(dv, dy, fw32[3 * b + 1]);
        fw32[3 * b + 2] = fmaf(dv, dz, fw32[3 * b + 2]);
      }
#pragma unroll
      for (int c = 0; c < 3; c++) gi[c] = warp_sumf(gi[c]);
      if (lane == 0) atomic_add3(P.d, A.atom, (double)gi[0], (double)gi[1], (double)gi[2]);
      continue;
    }
    if (act) {
#pragma unroll
      for (int b = 0; b < 3; b++) {
        double dx = xw[b].x - xi.x, dy = xw[b].y - xi.y, dz = xw[b].z - xi.z;
        double r = rsqrt(dx * dx + dy * dy + dz * dz);
        double r2 = r * r, r6 = r2 * r2 * r2;
        double Vel = (double)(b == 0 ? A.q.x : A.q.y) * r;
        double Va = (b == 0 ? A.lj.x : A.lj.z) * r6 * r6, Vb = (b == 0 ? A.lj.y : A.lj.w) * r6;
        double dv = r2 * (-Vel - 12. * Va + 6. * Vb);
        fi[0] -= dv * dx; fi[1] -= dv * dy; fi[2] -= dv * dz;
        fw[3 * b] += dv * dx; fw[3 * b + 1] += dv * dy; fw[3 * b + 2] += dv * dz;
        el += Vel;
        vdw += Va - Vb;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) fi[c] = warp_sum(fi[c]);
    if (lane == 0) atomic_add3(P.d, A.atom, fi[0], fi[1], fi[2]);
  }
  if (F32)
#pragma unroll
    for (int c = 0; c < 9; c++) fw[c] = (double)fw32[c];
  if (act)
    for (int b = 0; b < 3; b++) atomic_add3(P.d, o + b, fw[3 * b], fw[3 * b + 1], fw[3 * b + 2]);
  if (!F32) {
    warp_add(&P.E[s * QB_NE + QB_E_PW_EL], el);
    warp_add(&P.E[s * QB_NE + QB_E_PW_VDW], vdw);
  }
}

// nonbond_qp (md.f90:10980) / nonbond_qp_qvdw (11138): one thread per pair,
// all states in the thread.
template <int NSC>
__device__ __forceinline__ void nb_qp_body(DevPtrs &P, int bx, int s, int gx) {
  const SysDev &S = P.sys[s];
  int n = P.st[s].qp_n;
  const int NS = NSC > 0 ? NSC : S.S;
  const int ncol = S.natyps + S.nq;
  constexpr int NA = NSC > 0 ? NSC : MAXS;
  double el[NA], vdw[NA];
#pragma unroll
  for (int st = 0; st < NA; st++) { el[st] = 0; vdw[st] = 0; }
  for (int k0 = bx * blockDim.x; k0 < n; k0 += gx * blockDim.x) {
    int k = k0 + threadIdx.x;
    if (k < n) {
      int4 p = P.qp[S.qp_off + k];
      int gq = p.x, j = p.y, lj = p.z, qlj = p.w;
      int i = P.iqseq[gq], iq = gq - S.qoff;
      double3 xi = ld3(P.x, i), xj = ld3(P.x, j);
      double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
      if (S.pbc) {
        // nonbond_qp_box (md.f90:11060-11068): the image of j's group
        // switching atom nearest the Q switching atom
        const double3 a = ld3(P.x, S.qswitch), b = ld3(P.x, switch_of(P, j));
        const double3 t = image_shift(box_of(P, s), b.x - a.x, b.y - a.y, b.z - a.z);
        dx -= t.x; dy -= t.y; dz -= t.z;
      }
      double r2 = dx * dx + dy * dy + dz * dz;
      double dvsum = 0;
      if (!S.qvdw) {
        double r = rsqrt(r2);
        r2 = r * r;
        double r6 = r2 * r2 * r2;
        double aLJ, bLJ;
        lj_pair(S.arith, P.lja[3 * i + lj - 1], P.lja[3 * j + lj - 1], P.ljb[3 * i + lj - 1], P.ljb[3 * j + lj - 1],
                aLJ, bLJ);
        for (int st = 0; st < NS; st++) {
          float qq = P.qcrg[gq * MAXS + st] * P.crg[j];
          double Vel = (double)qq * r;
          if (lj == 3) Vel = Vel * S.el14;
          double Va = aLJ * r6 * r6, Vb = bLJ * r6;
          dvsum += r2 * (-Vel - 12. * Va + 6. * Vb) * S.lambda[st];
          el[st] += Vel;
          vdw[st] += Va - Vb;
        }
      } else {
        double r6 = r2 * r2 * r2;
        double r = rsqrt(r2);
        r2 = r * r;
        int tj = P.iac[j];
        for (int st = 0; st < NS; st++) {
          int ti = P.qiac[gq * MAXS + st];
          double aLJ, bLJ;
          lj_pair(S.arith, P.qavdw[S.qlib_off + 3 * ti + qlj - 1], P.lja[3 * j + lj - 1],
                  P.qbvdw[S.qlib_off + 3 * ti + qlj - 1], P.ljb[3 * j + lj - 1], aLJ, bLJ);
          float qq = P.qcrg[gq * MAXS + st] * P.crg[j];
          double Vel = (double)qq * r;
          if (lj == 3) Vel = Vel * S.el14;
          double r6sc = r6 + P.sc[S.sc_off + ((size_t)iq * ncol + tj) * NS + st];
          double Va = aLJ / (r6sc * r6sc), Vb = bLJ / r6sc;
          dvsum += r2 * (-Vel - (12. * Va - 6. * Vb) * (r6 / r6sc)) * S.lambda[st];
          el[st] += Vel;
          vdw[st] += Va - Vb;
        }
      }
      atomic_add3(P.d, i, -dvsum * dx, -dvsum * dy, -dvsum * dz);
      atomic_add3(P.d, j, dvsum * dx, dvsum * dy, dvsum * dz);
    }
  }
  for (int st = 0; st < NS; st++) {
    warp_add(&P.EQ[((size_t)s * MAXS + st) * QB_NEQ + QB_EQ_QP_EL], el[st]);
    warp_add(&P.EQ[((size_t)s * MAXS + st) * QB_NEQ + QB_EQ_QP_VDW], vdw[st]);
  }
}

// nonbond_qw_spc (md.f90:11302): Q atoms with the listed waters, one thread
// per water, all Q atoms and states in the thread.  The Q atoms' positions
// and per-state parameters (charge products with the water O and H in single
// precision as crg_ow*qcrg, LJ products with the water O, soft-core shifts)
// are staged in shared memory once per block.  Q-atom gradients are reduced
// per warp, then per block in shared memory (NQ_SHARED atoms at most; global
// atomics beyond).
// With hydrogen LJ (nonbon2_qw, md.f90:9798; nonbond_qw_3atom, 11545) the two
// hydrogen sites add LJ with their own type's parameters and soft-core shift.
struct QwState { float qO, qH; double A, B, sc, AH, BH, scH; };

// F32 (with SHQ, without hydrogen LJ): the mixed engine's steps that record
// no energies take the forces alone in FP32, as its water-water kernel does.
template <int NSC, bool SHQ, bool HLJ, bool F32 = false>
__global__ void __launch_bounds__(128, SHQ ? 4 : 1) k_nb_qw(DevPtrs P) {
  constexpr int NA = NSC > 0 ? NSC : MAXS;
  const int2 tile = P.qw_tiles[blockIdx.x];   // (system, first list entry)
  const int s = tile.x;
  const SysDev &S = P.sys[s];
  __shared__ double fq[NQ_SHARED * 3];
  __shared__ double4 qx[NQ_SHARED];        // position; w: LJ code
  __shared__ double2 qab[NQ_SHARED];       // A, B with the water O (same in every state)
  __shared__ double2 qabH[NQ_SHARED];      // A, B with a water H (hydrogen LJ only)
  __shared__ QwState qst[NQ_SHARED * NA];
  if (S.nq == 0) return;
  const int n = P.st[s].qw_n;
  if (tile.y >= n) return;
  const int NS = NSC > 0 ? NSC : S.S, ncol = S.natyps + S.nq;
  const bool hlj = HLJ && S.hlj;           // this system's water hydrogens carry LJ
  const bool shq = SHQ;                    // every system's Q atoms fit the shared tables
  const int nqs = shq ? S.nq : 0;
  for (int t = threadIdx.x; t < NQ_SHARED * 3; t += blockDim.x) fq[t] = 0;
  for (int iq = threadIdx.x; iq < nqs; iq += blockDim.x) {
    int gq = S.qoff + iq, i = P.iqseq[gq];
    int lj = P.ljcod[S.ljoff + S.iac_ow * S.natyps + P.iac[i]];
    int ljh = hlj ? P.ljcod[S.ljoff + S.iac_hw * S.natyps + P.iac[i]] : 1;
    double4 x = P.x[i];
    x.w = (double)(lj + 4 * ljh);
    qx[iq] = x;
    double A0, B0, AH0 = 0, BH0 = 0;
    lj_pair(S.arith, P.lja[3 * i + lj - 1], S.aO[lj - 1], P.ljb[3 * i + lj - 1], S.bO[lj - 1], A0, B0);
    if (hlj) lj_pair(S.arith, P.lja[3 * i + ljh - 1], S.aH[ljh - 1], P.ljb[3 * i + ljh - 1], S.bH[ljh - 1], AH0, BH0);
    qab[iq] = make_double2(A0, B0);
    qabH[iq] = make_double2(AH0, BH0);
    for (int st = 0; st < NS; st++) {
      QwState q;
      float c = P.qcrg[gq * MAXS + st];
      q.qO = S.crg_ow * c;
      q.qH = S.crg_hw * c;
      int ti = P.qiac[gq * MAXS + st];
      lj_pair(S.arith, P.qavdw[S.qlib_off + 3 * ti], S.aO[lj - 1], P.qbvdw[S.qlib_off + 3 * ti], S.bO[lj - 1], q.A, q.B);
      q.sc = S.qvdw ? P.sc[S.sc_off + ((size_t)iq * ncol + S.iac_ow) * NS + st] : 0.0;
      q.AH = q.BH = q.scH = 0.0;
      if (hlj) {
        lj_pair(S.arith, P.qavdw[S.qlib_off + 3 * ti], S.aH[ljh - 1], P.qbvdw[S.qlib_off + 3 * ti], S.bH[ljh - 1], q.AH,
                q.BH);
        q.scH = S.qvdw ? P.sc[S.sc_off + ((size_t)iq * ncol + S.iac_hw) * NS + st] : 0.0;
      }
      qst[iq * NA + st] = q;
    }
  }
  __syncthreads();
  double el[NA], vdw[NA];
#pragma unroll
  for (int st = 0; st < NA; st++) { el[st] = 0; vdw[st] = 0; }
  const int k = tile.y + threadIdx.x;
  const bool act = k < n;
  const int j = act ? P.qw[S.qw_off + k] : P.qw[S.qw_off];
  double3 xO = ld3(P.x, j), xH1 = ld3(P.x, j + 1), xH2 = ld3(P.x, j + 2);
  if (S.pbc) {
    // nonbond_qw_spc_box (md.f90:11440-11446): the water at the image of its
    // O nearest the Q switching atom
    const double3 a = ld3(P.x, S.qswitch);
    const double3 t = image_shift(box_of(P, s), xO.x - a.x, xO.y - a.y, xO.z - a.z);
    xO.x -= t.x; xO.y -= t.y; xO.z -= t.z;
    xH1.x -= t.x; xH1.y -= t.y; xH1.z -= t.z;
    xH2.x -= t.x; xH2.y -= t.y; xH2.z -= t.z;
  }
  double fw[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  float fw32[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int iq = 0; iq < S.nq; iq++) {
    int gq = S.qoff + iq;
    if (F32 && SHQ && !HLJ) {
      // forces alone in FP32: differences of the FP64 positions rounded to
      // FP32, MUFU reciprocal square roots, the states' sums in FP32
      const double4 xi4 = qx[iq];
      const float o[3] = {(float)(xO.x - xi4.x), (float)(xO.y - xi4.y), (float)(xO.z - xi4.z)};
      const float h1[3] = {(float)(xH1.x - xi4.x), (float)(xH1.y - xi4.y), (float)(xH1.z - xi4.z)};
      const float h2[3] = {(float)(xH2.x - xi4.x), (float)(xH2.y - xi4.y), (float)(xH2.z - xi4.z)};
      const float r2O = fmaf(o[0], o[0], fmaf(o[1], o[1], o[2] * o[2]));
      const float rO = rsqrt_ftz(r2O);
      const float rH1 = rsqrt_ftz(fmaf(h1[0], h1[0], fmaf(h1[1], h1[1], h1[2] * h1[2])));
      const float rH2 = rsqrt_ftz(fmaf(h2[0], h2[0], fmaf(h2[1], h2[1], h2[2] * h2[2])));
      const float r2Oi = rO * rO, r2H1 = rH1 * rH1, r2H2 = rH2 * rH2;
      const float r6hc = r2O * r2O * r2O;
      float Va0 = 0.f, Vb0 = 0.f;
      if (!S.qvdw) {
        const float r6 = r2Oi * r2Oi * r2Oi;
        Va0 = (float)qab[iq].x * r6 * r6;
        Vb0 = (float)qab[iq].y * r6;
      }
      float dvO = 0.f, dvH1 = 0.f, dvH2 = 0.f;
#pragma unroll
      for (int st = 0; st < NA; st++) {
        if (st >= NS) break;
        const QwState q = qst[iq * NA + st];
        float Va = Va0, Vb = Vb0, fsc = 1.f;
        if (S.qvdw) {
          const float inv = 1.f / (r6hc + (float)q.sc);
          Va = (float)q.A * inv * inv;
          Vb = (float)q.B * inv;
          fsc = r6hc * inv;
        }
        const float lam = (float)S.lambda[st];
        dvO += r2Oi * (-q.qO * rO - (12.f * Va - 6.f * Vb) * fsc) * lam;
        dvH1 -= r2H1 * (q.qH * rH1) * lam;
        dvH2 -= r2H2 * (q.qH * rH2) * lam;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float qa = act ? -(dvO * o[c] + dvH1 * h1[c] + dvH2 * h2[c]) : 0.f;
        fw32[c] = fmaf(dvO, o[c], fw32[c]);
        fw32[3 + c] = fmaf(dvH1, h1[c], fw32[3 + c]);
        fw32[6 + c] = fmaf(dvH2, h2[c], fw32[6 + c]);
        const float t = warp_sumf(qa);
        if ((threadIdx.x & 31) == 0 && t != 0.f) atomicAdd(&fq[3 * iq + c], (double)t);
      }
      continue;
    }
    double4 xi4;
    int lj, ljh;
    double A0, B0, AH0 = 0, BH0 = 0;
    if (shq) {
      xi4 = qx[iq];
      lj = (int)xi4.w & 3;
      ljh = (int)xi4.w >> 2;
      A0 = qab[iq].x; B0 = qab[iq].y;
      AH0 = qabH[iq].x; BH0 = qabH[iq].y;
    } else {
      int i = P.iqseq[gq];
      xi4 = P.x[i];
      lj = P.ljcod[S.ljoff + S.iac_ow * S.natyps + P.iac[i]];
      ljh = hlj ? P.ljcod[S.ljoff + S.iac_hw * S.natyps + P.iac[i]] : 1;
      lj_pair(S.arith, P.lja[3 * i + lj - 1], S.aO[lj - 1], P.ljb[3 * i + lj - 1], S.bO[lj - 1], A0, B0);
      if (hlj)
        lj_pair(S.arith, P.lja[3 * i + ljh - 1], S.aH[ljh - 1], P.ljb[3 * i + ljh - 1], S.bH[ljh - 1], AH0, BH0);
    }
    double dO[3] = {xO.x - xi4.x, xO.y - xi4.y, xO.z - xi4.z};
    double dH1[3] = {xH1.x - xi4.x, xH1.y - xi4.y, xH1.z - xi4.z};
    double dH2[3] = {xH2.x - xi4.x, xH2.y - xi4.y, xH2.z - xi4.z};
    double r2O = dO[0] * dO[0] + dO[1] * dO[1] + dO[2] * dO[2];
    double rH1 = rsqrt(dH1[0] * dH1[0] + dH1[1] * dH1[1] + dH1[2] * dH1[2]);
    double rH2 = rsqrt(dH2[0] * dH2[0] + dH2[1] * dH2[1] + dH2[2] * dH2[2]);
    double r6hc = r2O * r2O * r2O;
    double rO = rsqrt(r2O);
    r2O = rO * rO;
    double r2H1 = rH1 * rH1, r2H2 = rH2 * rH2;
    double dvO = 0, dvH1 = 0, dvH2 = 0, Va = 0, Vb = 0;
    if (!S.qvdw) {
      double r6O = 1. / r6hc;
      Va = A0 * r6O * r6O;
      Vb = B0 * r6O;
    }
    // hydrogen sites: d^6 and the hard-core LJ terms (state independent without qvdw)
    double d6H1 = 0, d6H2 = 0, VaH1 = 0, VbH1 = 0, VaH2 = 0, VbH2 = 0;
    if (hlj) {
      double r6H1 = r2H1 * r2H1 * r2H1, r6H2 = r2H2 * r2H2 * r2H2;
      d6H1 = 1. / r6H1; d6H2 = 1. / r6H2;
      if (!S.qvdw) {
        VaH1 = AH0 * r6H1 * r6H1; VbH1 = BH0 * r6H1;
        VaH2 = AH0 * r6H2 * r6H2; VbH2 = BH0 * r6H2;
      }
    }
#pragma unroll
    for (int st = 0; st < NA; st++) {
      if (st >= NS) break;
      QwState q;
      if (shq) q = qst[iq * NA + st];
      else {
        float c = P.qcrg[gq * MAXS + st];
        q.qO = S.crg_ow * c; q.qH = S.crg_hw * c;
        int ti = P.qiac[gq * MAXS + st];
        lj_pair(S.arith, P.qavdw[S.qlib_off + 3 * ti], S.aO[lj - 1], P.qbvdw[S.qlib_off + 3 * ti], S.bO[lj - 1], q.A,
                q.B);
        q.sc = S.qvdw ? P.sc[S.sc_off + ((size_t)iq * ncol + S.iac_ow) * NS + st] : 0.0;
        q.AH = q.BH = q.scH = 0.0;
        if (hlj) {
          lj_pair(S.arith, P.qavdw[S.qlib_off + 3 * ti], S.aH[ljh - 1], P.qbvdw[S.qlib_off + 3 * ti], S.bH[ljh - 1],
                  q.AH, q.BH);
          q.scH = S.qvdw ? P.sc[S.sc_off + ((size_t)iq * ncol + S.iac_hw) * NS + st] : 0.0;
        }
      }
      double r6sc = r6hc;
      if (S.qvdw) {
        r6sc = r6hc + q.sc;
        Va = q.A / (r6sc * r6sc);
        Vb = q.B / r6sc;
      }
      double VelO = (double)q.qO * rO;
      double VelH1 = (double)q.qH * rH1;
      double VelH2 = (double)q.qH * rH2;
      double lam = S.lambda[st];
      dvO += r2O * (-VelO - ((12. * Va - 6. * Vb) * (r6hc / r6sc))) * lam;
      if (hlj) {
        double f1 = 1.0, f2 = 1.0;
        if (S.qvdw) {
          double s1 = d6H1 + q.scH, s2 = d6H2 + q.scH;
          VaH1 = q.AH / (s1 * s1); VbH1 = q.BH / s1;
          VaH2 = q.AH / (s2 * s2); VbH2 = q.BH / s2;
          f1 = d6H1 / s1; f2 = d6H2 / s2;
        }
        dvH1 += r2H1 * (-VelH1 - (12. * VaH1 - 6. * VbH1) * f1) * lam;
        dvH2 += r2H2 * (-VelH2 - (12. * VaH2 - 6. * VbH2) * f2) * lam;
        if (act) vdw[st] += VaH1 + VaH2 - VbH1 - VbH2;
      } else {
        dvH1 -= r2H1 * VelH1 * lam;
        dvH2 -= r2H2 * VelH2 * lam;
      }
      if (act) {
        el[st] += VelO + VelH1 + VelH2;
        vdw[st] += Va - Vb;
      }
    }
    double qacc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      qacc[c] = act ? -(dvO * dO[c] + dvH1 * dH1[c] + dvH2 * dH2[c]) : 0.0;
      fw[c] += dvO * dO[c];
      fw[3 + c] += dvH1 * dH1[c];
      fw[6 + c] += dvH2 * dH2[c];
    }
    // Q-atom gradient: warp reduction, then one shared (or global) atomic per warp
#pragma unroll
    for (int c = 0; c < 3; c++) {
      double t = warp_sum(qacc[c]);
      if ((threadIdx.x & 31) == 0 && t != 0.0) {
        if (shq) atomicAdd(&fq[3 * iq + c], t);
        else atomicAdd(&P.d[P.iqseq[gq]].x + c, t);
      }
    }
  }
  if (F32 && SHQ && !HLJ)
#pragma unroll
    for (int c = 0; c < 9; c++) fw[c] = (double)fw32[c];
  if (act)
    for (int a = 0; a < 3; a++) atomic_add3(P.d, j + a, fw[3 * a], fw[3 * a + 1], fw[3 * a + 2]);
  if (!(F32 && SHQ && !HLJ))
    for (int st = 0; st < NS; st++) {
      warp_add(&P.EQ[((size_t)s * MAXS + st) * QB_NEQ + QB_EQ_QW_EL], el[st]);
      warp_add(&P.EQ[((size_t)s * MAXS + st) * QB_NEQ + QB_EQ_QW_VDW], vdw[st]);
    }
  __syncthreads();
  for (int t = threadIdx.x; t < nqs * 3; t += blockDim.x)
    if (fq[t] != 0.0) atomicAdd(&P.d[P.iqseq[S.qoff + t / 3]].x + (t % 3), fq[t]);
}

// nonbond_qq (md.f90:10763): Q-Q and Q-to-bonded-neighbour pairs, all states.
// With qq_use_library_charges (nonbond_qq_lib_charges, md.f90:10872) a Q-Q
// pair takes both atoms' topology charges; Q-to-neighbour pairs keep the Q
// atom's state charge, except under the arithmetic rule, whose
// nonbon2_qq_lib_charges (md.f90:9494) takes crg(i) for every pair.  A Q-Q
// soft pair (LJ code 2 with Q types) is A exp(-B/r) with A and B products
// under either rule (nonbon2_qq, md.f90:9426).
__device__ __forceinline__ void nb_qq_body(DevPtrs &P, int s) {
  const SysDev &S = P.sys[s];
  const int NS = S.S, ncol = S.natyps + S.nq;
  for (int k0 = 0; k0 < S.nqq; k0 += blockDim.x) {
    int k = k0 + threadIdx.x;
    double Vel = 0, V = 0;
    int st = 0;
    bool qq_pair = false, act = k < S.nqq;
    if (act) {
      int4 e = P.qq[S.qq_off + k];
      int gq = e.x, j = e.y, gjq = e.z, lj = e.w & 0xff;
      st = e.w >> 8;
      int iq = gq - S.qoff;
      int jq = gjq >= 0 ? gjq - S.qoff : -1;
      int i = P.iqseq[gq];
      const bool lib = S.qq_lib && jq >= 0;
      double qi = S.qq_lib && (jq >= 0 || S.arith) ? (double)P.crg[i] : (double)P.qcrg[gq * MAXS + st], qj, aLJ, bLJ;
      double els = P.qq_el[S.qq_off + k];
      if (!S.qvdw) {
        lj_pair(S.arith, P.lja[3 * i + lj - 1], P.lja[3 * j + lj - 1], P.ljb[3 * i + lj - 1], P.ljb[3 * j + lj - 1],
                aLJ, bLJ);
        qj = jq >= 0 && !lib ? (double)P.qcrg[gjq * MAXS + st] : (double)P.crg[j];
      } else {
        int ti = P.qiac[gq * MAXS + st];
        double ai = P.qavdw[S.qlib_off + 3 * ti + lj - 1], bi = P.qbvdw[S.qlib_off + 3 * ti + lj - 1];
        if (jq >= 0) {
          int tj = P.qiac[gjq * MAXS + st];
          lj_pair(S.arith && lj != 2, ai, P.qavdw[S.qlib_off + 3 * tj + lj - 1], bi,
                  P.qbvdw[S.qlib_off + 3 * tj + lj - 1], aLJ, bLJ);
          qj = lib ? P.crg[j] : P.qcrg[gjq * MAXS + st];
        } else {
          if (lj == 2) { ai = P.qavdw[S.qlib_off + 3 * ti]; bi = P.qbvdw[S.qlib_off + 3 * ti]; }
          lj_pair(S.arith, ai, P.lja[3 * j + lj - 1], bi, P.ljb[3 * j + lj - 1], aLJ, bLJ);
          qj = P.crg[j];
        }
      }
      double3 xi = ld3(P.x, i), xj = ld3(P.x, j);
      double dx = xj.x - xi.x, dy = xj.y - xi.y, dz = xj.z - xi.z;
      double r2 = dx * dx + dy * dy + dz * dz;
      double r6hc = r2 * r2 * r2;
      // jq = -1 reads the reference's sc_lookup(iq, natyps+0, state)
      double r6 = r2 * r2 * r2 + P.sc[S.sc_off + ((size_t)iq * ncol + (S.natyps + jq)) * NS + st];
      r6 = 1. / r6;
      double r12 = r6 * r6;
      r2 = 1. / r2;
      double r = sqrt(r2);
      Vel = qi * qj * r * els;
      if (lj == 3) Vel = Vel * S.el14;
      double Va, Vb, dv;
      if (S.qvdw && jq >= 0 && lj == 2) {
        Va = aLJ * exp(-bLJ / r);
        Vb = 0.0;
        dv = r2 * (-Vel - bLJ * Va / r) * S.lambda[st];
      } else {
        Va = aLJ * r12;
        Vb = bLJ * r6;
        dv = r2 * (-Vel - (12. * Va - 6. * Vb) * r6hc * r6) * S.lambda[st];
      }
      V = Va - Vb;
      qq_pair = jq >= 0;
      atomic_add3(P.d, i, -dv * dx, -dv * dy, -dv * dz);
      atomic_add3(P.d, j, dv * dx, dv * dy, dv * dz);
      double *eq = &P.EQ[((size_t)s * MAXS + st) * QB_NEQ];
      atomicAdd(&eq[qq_pair ? QB_EQ_QQ_EL : QB_EQ_QP_EL], Vel);
      atomicAdd(&eq[qq_pair ? QB_EQ_QQ_VDW : QB_EQ_QP_VDW], V);
    }
  }
}

// Per-atom terms (blockIdx.y = system), one update of each atom's gradient:
//  - lrf_taylor (md.f90:3646): potential and field of the atom's own group
//    multipoles; the reference's phi2(9) and phi3(27) are read through the
//    index of their distinct component, in its order of terms;
//  - fix_shell / restrain_solvent (md.f90:1414, 14910): harmonic restraints of
//    excluded and shell atoms to their topology positions, and the radial
//    restraint of water O atoms (harmonic outside the boundary less the
//    thermal shift, Morse inside).
// One thread per solute atom; the water atoms' terms are added by
// k_pack_waters (water_terms).
struct LrfRec { double v[24]; };

__device__ __forceinline__ void lrf_load(const DevPtrs &P, int gc, LrfRec &L) {
  const double4 *L4 = reinterpret_cast<const double4 *>(P.lrf + (size_t)gc * LRF_STRIDE);
#pragma unroll
  for (int w = 0; w < 6; w++) {
    double4 q = L4[w];
    L.v[4 * w] = q.x; L.v[4 * w + 1] = q.y; L.v[4 * w + 2] = q.z; L.v[4 * w + 3] = q.w;
  }
}

// Taylor potential and field of one atom at xi, charge q: returns 0.5*q*V,
// subtracts q*df from g.
__device__ __forceinline__ double lrf_eval(const LrfRec &R, double3 xi, double q, double *g) {
  constexpr int i2[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
  constexpr int i3[27] = {0, 1, 2, 1, 3, 4, 2, 4, 5, 1, 3, 4, 3, 6, 7, 4, 7, 8, 2, 4, 5, 4, 7, 8, 5, 8, 9};
  const double *L = R.v;
  double dr[3] = {L[0] - xi.x, L[1] - xi.y, L[2] - xi.z};
  const double *p1 = L + 4, *p2 = L + 7, *p3 = L + 13;
  double V = L[3] + p1[0] * dr[0] + p1[1] * dr[1] + p1[2] * dr[2];
#pragma unroll
  for (int a = 0; a < 3; a++)
    V += 0.5 * (p2[i2[3 * a]] * dr[0] + p2[i2[3 * a + 1]] * dr[1] + p2[i2[3 * a + 2]] * dr[2]) * dr[a];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double df = p1[c] + p2[i2[3 * c]] * dr[0] + p2[i2[3 * c + 1]] * dr[1] + p2[i2[3 * c + 2]] * dr[2];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int o = 9 * c + 3 * a;
      df += 0.5 * (p3[i3[o]] * dr[0] + p3[i3[o + 1]] * dr[1] + p3[i3[o + 2]] * dr[2]) * dr[a];
    }
    g[c] -= q * df;
  }
  return 0.5 * q * V;
}

// Harmonic restraint of an excluded or shell atom to its topology position.
__device__ __forceinline__ void fix_shell_atom(const DevPtrs &P, const SysDev &S, int i, uint8_t fl, double3 xi,
                                               double *g, double &efix, double &eshell) {
  double fk = (fl & F_EXCL) ? S.fk_fix : S.fk_pshell;
  double dr[3] = {xi.x - P.xtop[3 * i], xi.y - P.xtop[3 * i + 1], xi.z - P.xtop[3 * i + 2]};
  double e = 0.5 * fk * (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
  if (fl & F_EXCL) efix += e;
  if (fl & F_SHELL) eshell += e;
  for (int k = 0; k < 3; k++) g[k] += fk * dr[k];
}

// Gradient contributions after the water pass are atomic adds: the force
// kernels of one step run concurrently.
__device__ __forceinline__ void add_grad(DevPtrs &P, int i, const double *g) {
  if (g[0] != 0 || g[1] != 0 || g[2] != 0) atomic_add3(P.d, i, g[0], g[1], g[2]);
}

// The per-atom terms of one water (O at o, positions x): LRF Taylor terms of
// its three atoms (one record), fixed/shell restraints, and the radial
// restraint of its O.  Gradients into g[3][3].
__device__ __forceinline__ void water_terms(const DevPtrs &P, const SysDev &S, int s, int o, const double3 *x,
                                            double g[3][3], double &elrf, double &efix, double &eshell,
                                            double &erad) {
  const uint8_t fo = P.flags[o];
  if (S.use_lrf && !((fo & P.flags[o + 1] & P.flags[o + 2]) & F_EXCL)) {
    LrfRec R;
    lrf_load(P, P.cgp[o], R);
#pragma unroll
    for (int a = 0; a < 3; a++)
      if (!(P.flags[o + a] & F_EXCL) && P.iq[o + a] < 0) elrf += lrf_eval(R, x[a], (double)P.crg[o + a], g[a]);
  }
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const uint8_t fl = P.flags[o + a];
    if (fl & (F_EXCL | F_SHELL)) fix_shell_atom(P, S, o + a, fl, x[a], g[a], efix, eshell);
  }
  // the solvent sphere's radial restraint (restrain_solvent; none in a periodic box)
  if (!(fo & F_EXCL) && !S.pbc) {
    const double shift = S.fk_ws != 0. ? sqrt((double)kBoltzF * P.st[s].Tfree / S.fk_ws) : 0.;
    double dr[3] = {x[0].x - S.xw[0], x[0].y - S.xw[1], x[0].z - S.xw[2]};
    double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
    double db = b - (S.rwat - shift), e, dv;
    if (db > 0) { e = 0.5 * S.fk_ws * db * db - S.Dwmz; dv = S.fk_ws * db / b; }
    else if (b > 0.0) {
      double fexp = exp(S.awmz * db);
      e = S.Dwmz * (fexp * fexp - 2. * fexp);
      dv = -2. * S.Dwmz * S.awmz * (fexp - fexp * fexp) / b;
    } else { e = 0; dv = 0; }
    erad += e;
    for (int k = 0; k < 3; k++) g[0][k] += dv * dr[k];
  }
}

__global__ void k_atom_terms(DevPtrs P) {
  int s = blockIdx.y;
  const SysDev &S = P.sys[s];
  double elrf = 0, efix = 0, eshell = 0, erad = 0;
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u < S.nsol) {
    const int i = S.aoff + u;
    const uint8_t fl = P.flags[i];
    const double3 xi = ld3(P.x, i);
    double g[3] = {0, 0, 0};
    if (S.use_lrf && !(fl & F_EXCL) && P.iq[i] < 0) {
      LrfRec R;
      lrf_load(P, P.cgp[i], R);
      elrf += lrf_eval(R, xi, (double)P.crg[i], g);
    }
    if (fl & (F_EXCL | F_SHELL)) fix_shell_atom(P, S, i, fl, xi, g, efix, eshell);
    add_grad(P, i, g);
  }
  warp_add(&P.E[s * QB_NE + QB_E_LRF], elrf);
  warp_add(&P.E[s * QB_NE + QB_E_RST_FIX], efix);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SHELL], eshell);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SOLVENT_RADIAL], erad);
}

// The water-water kernels' records of water gw: FP64 (x y z of O, H1, H2)
// in wrec for the FP64 kernel; FP32 (O as hi + lo, H offsets from O) in
// wrec32 for the packed and FP32 kernels of the mixed engine, whose FP64
// pass (its energy-recording steps) writes both.
template <bool MIXED>
__device__ __forceinline__ void put_wat_records(const DevPtrs &P, int gw, double4 a, double4 b, double4 c) {
  if (MIXED || P.wrec32) {
    float4 *r = P.wrec32 + (size_t)gw * WatRec<true>::words;
    float hx = (float)a.x, hy = (float)a.y, hz = (float)a.z;
    float lx = (float)(a.x - (double)hx), ly = (float)(a.y - (double)hy), lz = (float)(a.z - (double)hz);
    r[0] = make_float4(hx, hy, hz, lx);
    r[1] = make_float4(ly, lz, (float)(b.x - a.x), (float)(c.x - a.x));
    r[2] = make_float4((float)(b.y - a.y), (float)(c.y - a.y), (float)(b.z - a.z), (float)(c.z - a.z));
  }
  if (!MIXED) {
    double2 *rd = reinterpret_cast<double2 *>(P.wrec + (size_t)gw * WatRec<false>::words);
    rd[0] = make_double2(a.x, a.y); rd[1] = make_double2(a.z, b.x); rd[2] = make_double2(b.y, b.z);
    rd[3] = make_double2(c.x, c.y); rd[4] = make_double2(c.z, 0.0);
  }
}

// Water pass, one thread per water, the step's first force kernel: the
// position record of the water-water kernel (see WatRec), the polarisation
// angle and shell, and the per-atom terms of its three atoms (water_terms),
// stored as their first gradient contribution; thread i also zeroes the
// gradient of solute atom i (the grid covers the larger of the two counts).
template <bool MIXED>
__global__ void k_pack_waters(DevPtrs P) {
  const int2 tile = P.pk_tiles[blockIdx.x];   // (system, first water or solute atom)
  const int s = tile.x;
  const SysDev &S = P.sys[s];
  const int iw = tile.y + threadIdx.x;
  double elrf = 0, efix = 0, eshell = 0, erad = 0;
  if (iw < S.nsol) P.d[S.aoff + iw] = make_double4(0.0, 0.0, 0.0, 0.0);   // the solute's gradient zeroed
  if (iw < S.nwat) {
    int o = S.aoff + S.nsol + 3 * iw;
    double4 a = P.x[o], b = P.x[o + 1], c = P.x[o + 2];
    if (S.wpol && S.nshell > 0) watpol_angle(P, S, S.woff + iw, (P.flags[o] & F_EXCL) != 0, a, b, c);
    put_wat_records<MIXED>(P, S.woff + iw, a, b, c);
    const double3 x[3] = {make_double3(a.x, a.y, a.z), make_double3(b.x, b.y, b.z), make_double3(c.x, c.y, c.z)};
    double g[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    water_terms(P, S, s, o, x, g, elrf, efix, eshell, erad);
#pragma unroll
    for (int k = 0; k < 3; k++) P.d[o + k] = make_double4(g[k][0], g[k][1], g[k][2], 0.0);
  }
  warp_add(&P.E[s * QB_NE + QB_E_LRF], elrf);
  warp_add(&P.E[s * QB_NE + QB_E_RST_FIX], efix);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SHELL], eshell);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SOLVENT_RADIAL], erad);
}

// The water pass with one thread per water atom (the same terms in the same
// order per atom; the O's thread adds the radial restraint, the first H's the
// polarisation angle, the second H's the water's record): three times the
// threads of k_pack_waters for batches too small to fill the GPU with one
// thread per water.
template <bool MIXED>
__global__ void k_pack_water_atoms(DevPtrs P) {
  int s = blockIdx.y;
  const SysDev &S = P.sys[s];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int iw = t / 3, a = t - 3 * iw;     // water, and its atom this thread takes
  double elrf = 0, efix = 0, eshell = 0, erad = 0;
  if (t < S.nsol) P.d[S.aoff + t] = make_double4(0.0, 0.0, 0.0, 0.0);   // the solute's gradient zeroed
  if (iw < S.nwat) {
    const int o = S.aoff + S.nsol + 3 * iw, i = o + a;
    const double4 xa4 = P.x[i];
    const double3 xa = make_double3(xa4.x, xa4.y, xa4.z);
    if (a == 1 && S.wpol && S.nshell > 0)
      watpol_angle(P, S, S.woff + iw, (P.flags[o] & F_EXCL) != 0, P.x[o], xa4, P.x[o + 2]);
    if (a == 2) put_wat_records<MIXED>(P, S.woff + iw, P.x[o], P.x[o + 1], xa4);
    double g[3] = {0, 0, 0};
    const uint8_t fo = P.flags[o], fl = P.flags[i];
    if (S.use_lrf && !((fo & P.flags[o + 1] & P.flags[o + 2]) & F_EXCL) && !(fl & F_EXCL) && P.iq[i] < 0) {
      LrfRec R;
      lrf_load(P, P.cgp[o], R);
      elrf += lrf_eval(R, xa, (double)P.crg[i], g);
    }
    if (fl & (F_EXCL | F_SHELL)) fix_shell_atom(P, S, i, fl, xa, g, efix, eshell);
    // the solvent sphere's radial restraint on the O (restrain_solvent; none in a periodic box)
    if (a == 0 && !(fo & F_EXCL) && !S.pbc) {
      const double shift = S.fk_ws != 0. ? sqrt((double)kBoltzF * P.st[s].Tfree / S.fk_ws) : 0.;
      double dr[3] = {xa.x - S.xw[0], xa.y - S.xw[1], xa.z - S.xw[2]};
      double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      double db = b - (S.rwat - shift), e, dv;
      if (db > 0) { e = 0.5 * S.fk_ws * db * db - S.Dwmz; dv = S.fk_ws * db / b; }
      else if (b > 0.0) {
        double fexp = exp(S.awmz * db);
        e = S.Dwmz * (fexp * fexp - 2. * fexp);
        dv = -2. * S.Dwmz * S.awmz * (fexp - fexp * fexp) / b;
      } else { e = 0; dv = 0; }
      erad += e;
      for (int k = 0; k < 3; k++) g[k] += dv * dr[k];
    }
    P.d[i] = make_double4(g[0], g[1], g[2], 0.0);
  }
  warp_add(&P.E[s * QB_NE + QB_E_LRF], elrf);
  warp_add(&P.E[s * QB_NE + QB_E_RST_FIX], efix);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SHELL], eshell);
  warp_add(&P.E[s * QB_NE + QB_E_RST_SOLVENT_RADIAL], erad);
}

// ---------------------------------------------------------------- bonded

__device__ __forceinline__ double dihedral(const DevPtrs &P, int i, int j, int k, int l, double dp[12]) {
  double3 xi = ld3(P.x, i), xj = ld3(P.x, j), xk = ld3(P.x, k), xl = ld3(P.x, l);
  double rji[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
  double rjk[3] = {xk.x - xj.x, xk.y - xj.y, xk.z - xj.z};
  double rkl[3] = {xl.x - xk.x, xl.y - xk.y, xl.z - xk.z};
  double rnj[3], rnk[3], di[3], dl[3], rki[3], rlj[3];
  rnj[0] = rji[1] * rjk[2] - rji[2] * rjk[1];
  rnj[1] = rji[2] * rjk[0] - rji[0] * rjk[2];
  rnj[2] = rji[0] * rjk[1] - rji[1] * rjk[0];
  rnk[0] = -rjk[1] * rkl[2] + rjk[2] * rkl[1];
  rnk[1] = -rjk[2] * rkl[0] + rjk[0] * rkl[2];
  rnk[2] = -rjk[0] * rkl[1] + rjk[1] * rkl[0];
  double bj2inv = 1. / (rnj[0] * rnj[0] + rnj[1] * rnj[1] + rnj[2] * rnj[2]);
  double bk2inv = 1. / (rnk[0] * rnk[0] + rnk[1] * rnk[1] + rnk[2] * rnk[2]);
  double bjinv = sqrt(bj2inv), bkinv = sqrt(bk2inv);
  double scp = (rnj[0] * rnk[0] + rnj[1] * rnk[1] + rnj[2] * rnk[2]) * (bjinv * bkinv);
  double phi;
  if (scp > 1.0) { scp = 1.0; phi = (double)acosf(1.0f); }
  else if (scp < -1.0) { scp = -1.0; phi = (double)acosf(-1.0f); }
  else phi = acos(scp);
  double sgn = rjk[0] * (rnj[1] * rnk[2] - rnj[2] * rnk[1]) + rjk[1] * (rnj[2] * rnk[0] - rnj[0] * rnk[2]) +
               rjk[2] * (rnj[0] * rnk[1] - rnj[1] * rnk[0]);
  if (sgn < 0) phi = -phi;
  double f1 = sin(phi);
  if (fabs(f1) < 1.e-12) f1 = 1.e-12;
  f1 = -1.0 / f1;
  for (int c = 0; c < 3; c++) {
    di[c] = f1 * (rnk[c] * (bjinv * bkinv) - scp * rnj[c] * bj2inv);
    dl[c] = f1 * (rnj[c] * (bjinv * bkinv) - scp * rnk[c] * bk2inv);
    rki[c] = rji[c] - rjk[c];
    rlj[c] = -rjk[c] - rkl[c];
  }
  dp[0] = rjk[1] * di[2] - rjk[2] * di[1];
  dp[1] = rjk[2] * di[0] - rjk[0] * di[2];
  dp[2] = rjk[0] * di[1] - rjk[1] * di[0];
  dp[3] = rki[1] * di[2] - rki[2] * di[1] + rkl[1] * dl[2] - rkl[2] * dl[1];
  dp[4] = rki[2] * di[0] - rki[0] * di[2] + rkl[2] * dl[0] - rkl[0] * dl[2];
  dp[5] = rki[0] * di[1] - rki[1] * di[0] + rkl[0] * dl[1] - rkl[1] * dl[0];
  dp[6] = rlj[1] * dl[2] - rlj[2] * dl[1] - rji[1] * di[2] + rji[2] * di[1];
  dp[7] = rlj[2] * dl[0] - rlj[0] * dl[2] - rji[2] * di[0] + rji[0] * di[2];
  dp[8] = rlj[0] * dl[1] - rlj[1] * dl[0] - rji[0] * di[1] + rji[1] * di[0];
  dp[9] = rjk[1] * dl[2] - rjk[2] * dl[1];
  dp[10] = rjk[2] * dl[0] - rjk[0] * dl[2];
  dp[11] = rjk[0] * dl[1] - rjk[1] * dl[0];
  return phi;
}

__device__ __forceinline__ void apply4(const DevPtrs &P, int i, int j, int k, int l, double dv, const double dp[12]) {
  atomic_add3(P.d, i, dv * dp[0], dv * dp[1], dv * dp[2]);
  atomic_add3(P.d, j, dv * dp[3], dv * dp[4], dv * dp[5]);
  atomic_add3(P.d, k, dv * dp[6], dv * dp[7], dv * dp[8]);
  atomic_add3(P.d, l, dv * dp[9], dv * dp[10], dv * dp[11]);
}

// bond (954), angle (814), torsion (14793), improper (1677) / improper2 (1789):
// one thread per term; items are bonds, then angles, torsions, impropers.
__device__ __forceinline__ void bonded_body(DevPtrs &P, int bx, int s, int gx) {
  const SysDev &S = P.sys[s];
  int n = S.nb + S.na + S.nt + S.ni;
  double e[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // p bond, angle, torsion, improper; w ...
  const double pi = dev_pi();
  for (int k0 = bx * blockDim.x; k0 < n; k0 += gx * blockDim.x) {
    int k = k0 + threadIdx.x;
    if (k >= n) continue;
    if (k < S.nb) {
      int2 b = P.bij[S.b_off + k];
      double2 prm = P.bpar[S.b_off + k];
      double3 xi = ld3(P.x, b.x), xj = ld3(P.x, b.y);
      double r[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
      double bl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      double db = bl - prm.y;
      e[k < S.nb_sol ? 0 : 4] += 0.5 * prm.x * db * db;
      double dv = prm.x * db / bl;
      atomic_add3(P.d, b.y, r[0] * dv, r[1] * dv, r[2] * dv);
      atomic_add3(P.d, b.x, -r[0] * dv, -r[1] * dv, -r[2] * dv);
    } else if (k < S.nb + S.na) {
      int a = k - S.nb;
      int4 t = P.aijk[S.a_off + a];
      double2 prm = P.apar[S.a_off + a];
      double3 xi = ld3(P.x, t.x), xj = ld3(P.x, t.y), xk = ld3(P.x, t.z);
      double rji[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
      double rjk[3] = {xk.x - xj.x, xk.y - xj.y, xk.z - xj.z};
      double bji2inv = 1. / (rji[0] * rji[0] + rji[1] * rji[1] + rji[2] * rji[2]);
      double bjk2inv = 1. / (rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
      double bjiinv = sqrt(bji2inv), bjkinv = sqrt(bjk2inv);
      double scp = (rji[0] * rjk[0] + rji[1] * rjk[1] + rji[2] * rjk[2]) * bjiinv * bjkinv;
      if (scp > 1.0) scp = 1.0;
      else if (scp < -1.0) scp = -1.0;
      double ang = acos(scp);
      double da = ang - prm.y;
      e[a < S.na_sol ? 1 : 5] += 0.5 * prm.x * da * da;
      double dv = prm.x * da;
      double f1 = sin(ang);
      if (fabs(f1) < 1.e-12) f1 = -1.e12;
      else f1 = -1.0 / f1;
      double di[3], dk[3];
      for (int c = 0; c < 3; c++) {
        di[c] = f1 * (rjk[c] * bjiinv * bjkinv - scp * rji[c] * bji2inv);
        dk[c] = f1 * (rji[c] * bjiinv * bjkinv - scp * rjk[c] * bjk2inv);
      }
      atomic_add3(P.d, t.x, dv * di[0], dv * di[1], dv * di[2]);
      atomic_add3(P.d, t.z, dv * dk[0], dv * dk[1], dv * dk[2]);
      atomic_add3(P.d, t.y, -dv * (di[0] + dk[0]), -dv * (di[1] + dk[1]), -dv * (di[2] + dk[2]));
      if (S.ff_type == 3) {  // urey_bradley (md.f90:904): harmonic 1-3 distance, k r^2 without 1/2
        double2 ub = P.aub[S.a_off + a];
        if (ub.x > 0.) {
          double rik[3] = {xk.x - xi.x, xk.y - xi.y, xk.z - xi.z};
          double dik = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]);
          double ru = dik - ub.y;
          e[a < S.na_sol ? 1 : 5] += ub.x * ru * ru;
          double du = 2. * ub.x * ru / dik;
          atomic_add3(P.d, t.z, du * rik[0], du * rik[1], du * rik[2]);
          atomic_add3(P.d, t.x, -du * rik[0], -du * rik[1], -du * rik[2]);
        }
      }
    } else if (k < S.nb + S.na + S.nt) {
      int t = k - S.nb - S.na;
      int4 q = P.tijkl[S.t_off + t];
      float4 prm = P.tpar[S.t_off + t];  // fk, rmult, deltor, paths
      double dp[12];
      double phi = dihedral(P, q.x, q.y, q.z, q.w, dp);
      double arg = (double)prm.y * phi - (double)prm.z;
      e[t < S.nt_sol ? 2 : 6] += (double)prm.x * (1.0 + cos(arg)) * (double)prm.w;
      float rf = prm.y * prm.x;
      double dv = -((double)rf * sin(arg) * (double)prm.w);
      apply4(P, q.x, q.y, q.z, q.w, dv, dp);
    } else {
      int t = k - S.nb - S.na - S.nt;
      int4 q = P.iijkl[S.i_off + t];
      float2 prm = P.ipar[S.i_off + t];  // fk, imp0
      double dp[12];
      double phi = dihedral(P, q.x, q.y, q.z, q.w, dp);
      double dv, ee;
      if (S.ff_type == 2) {
        double arg = 2 * phi - (double)prm.y;
        ee = (double)prm.x * (1 + cos(arg));
        dv = -2 * (double)prm.x * sin(arg);
      } else {
        double arg = phi - (double)prm.y;
        arg = arg - 2. * pi * (double)llround(arg / (2. * pi));
        dv = (double)prm.x * arg;
        ee = 0.5 * dv * arg;
      }
      e[t < S.ni_sol ? 3 : 7] += ee;
      apply4(P, q.x, q.y, q.z, q.w, dv, dp);
    }
  }
  const int idx[8] = {QB_E_P_BOND, QB_E_P_ANGLE, QB_E_P_TORSION, QB_E_P_IMPROPER,
                      QB_E_W_BOND, QB_E_W_ANGLE, QB_E_W_TORSION, QB_E_W_IMPROPER};
  for (int c = 0; c < 8; c++) warp_add(&P.E[s * QB_NE + idx[c]], e[c]);
}

// EMorseD of Q bond qb (global index) as qbond computed it in state st, and
// dMorse_i (dMorse_j = -dMorse_i), md.f90:14086-14108: the Morse bond's
// fraction of its well depth beyond r0, 1 inside it.
__device__ __forceinline__ double morse_gamma(const DevPtrs &P, const SysDev &S, int qb, int st, double *dmi,
                                              int2 &ij) {
  ij = P.qbij[qb];
  const double4 prm = P.qbpar[qb * MAXS + st];   // Dmz, amz, r0, fk
  const double3 xi = ld3(P.x, ij.x), xj = ld3(P.x, ij.y);
  const double r[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
  const double b = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  const double db = b - prm.z;
  const double fexp = exp(-prm.y * db);
  if (db > 0) {
    const double f = 2. * prm.y * (fexp - fexp * fexp) * S.lambda[st] / b;
    for (int c = 0; c < 3; c++) dmi[c] = f * r[c];
    return -(fexp * fexp - 2. * fexp);
  }
  dmi[0] = dmi[1] = dmi[2] = 0.0;
  return 1.0;
}

// The coupling's gradient: dMorse_i * E on the bond's first atom, dMorse_j * E
// on its second (md.f90:13970-13985).
__device__ __forceinline__ void morse_apply(DevPtrs &P, int2 ij, const double *dmi, double e) {
  atomic_add3(P.d, ij.x, dmi[0] * e, dmi[1] * e, dmi[2] * e);
  atomic_add3(P.d, ij.y, -dmi[0] * e, -dmi[1] * e, -dmi[2] * e);
}

// qbond (14060), qangle (13896), qtorsion (14262), qimproper (14117):
// one block per system, threads over (term, state).  A term coupled to a
// Morse bond (EVB couplings) is scaled by gamma = EMorseD of that bond, with
// the bond's values from the state qbond last set them in (setup resolves it).
__device__ __forceinline__ void qbonded_body(DevPtrs &P, int s) {
  const SysDev &S = P.sys[s];
  // offdiag (md.f90:12911): the Q-atom distance of each off-diagonal
  // function, from this step's coordinates; Hij = A exp(-mu r) is formed on
  // the host where the records are written
  if ((int)threadIdx.x < S.noffd) {
    double3 a = ld3(P.x, S.offd_k[threadIdx.x]), b = ld3(P.x, S.offd_l[threadIdx.x]);
    P.offd_r[s * MAXS + threadIdx.x] =
        sqrt((b.x - a.x) * (b.x - a.x) + (b.y - a.y) * (b.y - a.y) + (b.z - a.z) * (b.z - a.z));
  }
  const int NS = S.S;
  int n1 = S.nqb * NS, n2 = n1 + S.nqa * NS, n3 = n2 + S.nqt * NS, n4 = n3 + S.nqi * NS;
  const double pi = dev_pi();
  for (int k = threadIdx.x; k < n4; k += blockDim.x) {
    double *eq;
    if (k < n1) {
      int b = k / NS, st = k % NS;
      if (!P.qb_on[(S.qb_off + b) * MAXS + st]) continue;
      eq = &P.EQ[((size_t)s * MAXS + st) * QB_NEQ];
      int2 ij = P.qbij[S.qb_off + b];
      double4 prm = P.qbpar[(S.qb_off + b) * MAXS + st];  // Dmz, amz, r0, fk
      double3 xi = ld3(P.x, ij.x), xj = ld3(P.x, ij.y);
      double r[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
      double bl = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      double db = bl - prm.z;
      double fexp = exp(-prm.y * db);
      atomicAdd(&eq[QB_EQ_BOND], prm.x * (fexp * fexp - 2. * fexp) + 0.5 * prm.w * db * db);
      double dv = (2. * prm.x * prm.y * (fexp - fexp * fexp) + prm.w * db) * S.lambda[st] / bl;
      atomic_add3(P.d, ij.x, -dv * r[0], -dv * r[1], -dv * r[2]);
      atomic_add3(P.d, ij.y, dv * r[0], dv * r[1], dv * r[2]);
    } else if (k < n2) {
      int a = (k - n1) / NS, st = (k - n1) % NS;
      if (!P.qa_on[(S.qa_off + a) * MAXS + st]) continue;
      eq = &P.EQ[((size_t)s * MAXS + st) * QB_NEQ];
      int4 t = P.qaijk[S.qa_off + a];
      double2 prm = P.qapar[(S.qa_off + a) * MAXS + st];
      double3 xi = ld3(P.x, t.x), xj = ld3(P.x, t.y), xk = ld3(P.x, t.z);
      double rji[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
      double rjk[3] = {xk.x - xj.x, xk.y - xj.y, xk.z - xj.z};
      double bji = sqrt(rji[0] * rji[0] + rji[1] * rji[1] + rji[2] * rji[2]);
      double bjk = sqrt(rjk[0] * rjk[0] + rjk[1] * rjk[1] + rjk[2] * rjk[2]);
      double scp = (rji[0] * rjk[0] + rji[1] * rjk[1] + rji[2] * rjk[2]) / (bji * bjk);
      if (scp > 1.0) scp = 1.0;
      if (scp < -1.0) scp = -1.0;
      double ang = acos(scp);
      double da = ang - prm.y;
      const int2 cp = P.qa_cpl[S.qa_off + a];
      double gamma = 1.0, dmi[3];
      int2 bij;
      if (cp.x >= 0) gamma = morse_gamma(P, S, cp.x, P.qa_src[(S.qa_off + a) * MAXS + st], dmi, bij);
      const double ae = 0.5 * prm.x * da * da;
      atomicAdd(&eq[QB_EQ_ANGLE], ae * gamma);
      double dv = gamma * prm.x * da * S.lambda[st];
      double f1 = sin(ang);
      if (fabs(f1) < 1.e-12) f1 = 1.e-12;
      f1 = -1.0 / f1;
      double di[3], dk[3];
      for (int c = 0; c < 3; c++) {
        di[c] = f1 * (rjk[c] / (bji * bjk) - scp * rji[c] / (bji * bji));
        dk[c] = f1 * (rji[c] / (bji * bjk) - scp * rjk[c] / (bjk * bjk));
      }
      atomic_add3(P.d, t.x, dv * di[0], dv * di[1], dv * di[2]);
      atomic_add3(P.d, t.z, dv * dk[0], dv * dk[1], dv * dk[2]);
      atomic_add3(P.d, t.y, -dv * (di[0] + dk[0]), -dv * (di[1] + dk[1]), -dv * (di[2] + dk[2]));
      if (cp.x >= 0) morse_apply(P, bij, dmi, ae);
      // qurey_bradley (md.f90:13992): adds the 1-3 energy to the state's
      // angle energy; the reference never applies its gradient, so neither
      // does this (a Morse coupling's gradient it does apply)
      double2 ub = P.qaub[(S.qa_off + a) * MAXS + st];
      if (ub.x != 0.) {
        double rik[3] = {xk.x - xi.x, xk.y - xi.y, xk.z - xi.z};
        double ru = sqrt(rik[0] * rik[0] + rik[1] * rik[1] + rik[2] * rik[2]) - ub.y;
        const double eu = ub.x * ru * ru;
        double g = 1.0;
        if (cp.y >= 0) g = morse_gamma(P, S, cp.y, P.qa_src_ub[(S.qa_off + a) * MAXS + st], dmi, bij);
        atomicAdd(&eq[QB_EQ_ANGLE], eu * g);
        if (cp.y >= 0) morse_apply(P, bij, dmi, eu);
      }
    } else if (k < n3) {
      int t = (k - n2) / NS, st = (k - n2) % NS;
      if (!P.qt_on[(S.qt_off + t) * MAXS + st]) continue;
      eq = &P.EQ[((size_t)s * MAXS + st) * QB_NEQ];
      int4 q = P.qtijkl[S.qt_off + t];
      double4 prm = P.qtpar[(S.qt_off + t) * MAXS + st];  // fk, rmult, deltor
      double dp[12];
      double phi = dihedral(P, q.x, q.y, q.z, q.w, dp);
      double arg = prm.y * phi - prm.z;
      const int2 cp = P.qt_cpl[S.qt_off + t];
      double gamma = 1.0, dmi[3];
      int2 bij;
      if (cp.x >= 0) gamma = morse_gamma(P, S, cp.x, P.qt_src[(S.qt_off + t) * MAXS + st], dmi, bij);
      const double pe = prm.x * (1.0 + cos(arg));
      atomicAdd(&eq[QB_EQ_TORSION], pe * gamma);
      double dv = -prm.y * prm.x * sin(arg) * gamma * S.lambda[st];
      apply4(P, q.x, q.y, q.z, q.w, dv, dp);
      if (cp.x >= 0) morse_apply(P, bij, dmi, pe);
    } else {
      int t = (k - n3) / NS, st = (k - n3) % NS;
      if (!P.qi_on[(S.qi_off + t) * MAXS + st]) continue;
      eq = &P.EQ[((size_t)s * MAXS + st) * QB_NEQ];
      int4 q = P.qiijkl[S.qi_off + t];
      double2 prm = P.qipar[(S.qi_off + t) * MAXS + st];  // fk, imp0
      double dp[12];
      double phi = dihedral(P, q.x, q.y, q.z, q.w, dp);
      double arg = phi - prm.y;
      arg = arg - 2. * pi * (double)llround(arg / (2. * pi));
      const int2 cp = P.qi_cpl[S.qi_off + t];
      double gamma = 1.0, dmi[3];
      int2 bij;
      if (cp.x >= 0) {
        gamma = morse_gamma(P, S, cp.x, P.qi_src[(S.qi_off + t) * MAXS + st], dmi, bij);
        if (cp.y == 1) gamma = 1 - gamma;   // coupled to a bond breaking, not making
      }
      double dv = prm.x * arg;
      const double pe = 0.5 * dv * arg;
      atomicAdd(&eq[QB_EQ_IMPROPER], pe * gamma);
      dv = dv * gamma * S.lambda[st];
      apply4(P, q.x, q.y, q.z, q.w, dv, dp);
      if (cp.x >= 0) morse_apply(P, bij, dmi, pe);
    }
  }
}

// ------------------------------------------------------------ restraints


__device__ __forceinline__ double block_sum(double v, double *sh) {
  v = warp_sum(v);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0;
  for (int w = 0; w < nw; w++) t += sh[w];
  return t;
}

__device__ __forceinline__ void rst_energy(const DevPtrs &P, int s, int nstates, int ipsi, double e) {
  if (ipsi == 0) {
    for (int k = 0; k < nstates; k++) atomicAdd(&P.EQ[((size_t)s * MAXS + k) * QB_NEQ + QB_EQ_RESTRAINT], e);
    if (nstates == 0) atomicAdd(&P.E[s * QB_NE + QB_E_RST_PROTEIN], e);
  } else {
    atomicAdd(&P.EQ[((size_t)s * MAXS + ipsi - 1) * QB_NEQ + QB_EQ_RESTRAINT], e);
  }
}

// p_restrain (md.f90:12940): sequence, atom, distance, angle and wall
// restraints.  One block per system.
__device__ __forceinline__ void prestrain_body(DevPtrs &P, int s) {
  const SysDev &S = P.sys[s];
  __shared__ double sh[32];
  for (int r = 0; r < S.nrs; r++) {
    int4 q = P.rs[S.rs_off + r];  // i, j, ih, to_center
    double fk = P.rs_fk[S.rs_off + r];
    if (q.w == 1 || q.w == 2) {
      double acc[4] = {0, 0, 0, 0};
      for (int i = q.x + threadIdx.x; i <= q.y; i += blockDim.x) {
        if (!((P.flags[i] & F_HEAVY) || q.z == 1)) continue;
        double w = q.w == 2 ? P.mass[i] : 1.0;
        double3 xi = ld3(P.x, i);
        acc[0] += (xi.x - P.xtop[3 * i]) * w;
        acc[1] += (xi.y - P.xtop[3 * i + 1]) * w;
        acc[2] += (xi.z - P.xtop[3 * i + 2]) * w;
        acc[3] += w;
      }
      double tot[4];
      for (int k = 0; k < 4; k++) tot[k] = block_sum(acc[k], sh);
      if (tot[3] > 0) {
        double dr[3];
        for (int k = 0; k < 3; k++) dr[k] = tot[k] / tot[3];
        double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
        if (threadIdx.x == 0) atomicAdd(&P.E[s * QB_NE + QB_E_RST_PROTEIN], 0.5 * fk * r2);
        for (int i = q.x + threadIdx.x; i <= q.y; i += blockDim.x) {
          if (!((P.flags[i] & F_HEAVY) || q.z == 1)) continue;
          double sc = q.w == 1 ? fk * P.mass[i] / (double)12.010f : fk;
          atomic_add3(P.d, i, sc * dr[0], sc * dr[1], sc * dr[2]);
        }
      }
      __syncthreads();
    } else {
      double e = 0;
      for (int i = q.x + threadIdx.x; i <= q.y; i += blockDim.x) {
        if (!((P.flags[i] & F_HEAVY) || q.z == 1)) continue;
        double3 xi = ld3(P.x, i);
        double dr[3] = {xi.x - P.xtop[3 * i], xi.y - P.xtop[3 * i + 1], xi.z - P.xtop[3 * i + 2]};
        e += 0.5 * fk * (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
        atomic_add3(P.d, i, fk * dr[0], fk * dr[1], fk * dr[2]);
      }
      double t = block_sum(e, sh);
      if (threadIdx.x == 0) atomicAdd(&P.E[s * QB_NE + QB_E_RST_PROTEIN], t);
      __syncthreads();
    }
  }
  const double deg2rad = dev_pi() / 180.0;
  int nall = S.nrp + S.nrd + S.nra;
  for (int k = threadIdx.x; k < nall; k += blockDim.x) {
    if (k < S.nrp) {
      int2 q = P.rp[S.rp_off + k];  // i, ipsi
      const double *xr = P.rp_x + 3 * (S.rp_off + k), *fk = P.rp_fk + 3 * (S.rp_off + k);
      double3 xi = ld3(P.x, q.x);
      double dr[3] = {xi.x - xr[0], xi.y - xr[1], xi.z - xr[2]};
      double wgt = q.y != 0 ? S.lambda[q.y - 1] : 1.0, e = 0;
      for (int c = 0; c < 3; c++) e += 0.5 * fk[c] * dr[c] * dr[c];
      atomic_add3(P.d, q.x, fk[0] * dr[0] * wgt, fk[1] * dr[1] * wgt, fk[2] * dr[2] * wgt);
      rst_energy(P, s, S.S, q.y, e);
    } else if (k < S.nrp + S.nrd) {
      int r = k - S.nrp;
      int4 q = P.rd[S.rd_off + r];  // i, j, ipsi
      double4 prm = P.rd_p[S.rd_off + r];  // d1, d2, fk
      double3 xi = ld3(P.x, q.x), xj = ld3(P.x, q.y);
      double dr[3] = {xj.x - xi.x, xj.y - xi.y, xj.z - xi.z};
      if (S.pbc) min_image(box_of(P, s), dr[0], dr[1], dr[2]);   // md.f90:13096-13101
      double wgt = q.z != 0 ? S.lambda[q.z - 1] : 1.0;
      double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]), db;
      if (b < prm.x) db = b - prm.x;
      else if (b > prm.y) db = b - prm.y;
      else continue;
      double e = 0.5 * prm.z * db * db, dv = wgt * prm.z * db / b;
      atomic_add3(P.d, q.y, dr[0] * dv, dr[1] * dv, dr[2] * dv);
      atomic_add3(P.d, q.x, -dr[0] * dv, -dr[1] * dv, -dr[2] * dv);
      rst_energy(P, s, S.S, q.z, e);
    } else {
      int r = k - S.nrp - S.nrd;
      int4 q = P.ra[S.ra_off + r];  // i, j, k, ipsi
      double2 prm = P.ra_p[S.ra_off + r];  // ang, fk
      double3 xi = ld3(P.x, q.x), xj = ld3(P.x, q.y), xk = ld3(P.x, q.z);
      double d1[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z}, d2[3] = {xk.x - xj.x, xk.y - xj.y, xk.z - xj.z};
      if (S.pbc) {   // md.f90:13160-13168
        const BoxD bx = box_of(P, s);
        min_image(bx, d1[0], d1[1], d1[2]);
        min_image(bx, d2[0], d2[1], d2[2]);
      }
      double wgt = q.w != 0 ? S.lambda[q.w - 1] : 1.0;
      double r2ij = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2], r2jk = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
      double rij = sqrt(r2ij), rjk = sqrt(r2jk);
      double scp = (d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2]) / (rij * rjk);
      if (scp > 1.0) scp = 1.0;
      if (scp < -1.0) scp = -1.0;
      double th = acos(scp);
      double db = th - prm.x * deg2rad;
      double e = 0.5 * prm.y * db * db, dv = wgt * prm.y * db;
      double f1 = sin(th);
      if (fabs(f1) < 1.e-12) f1 = -1.e12;
      else f1 = -1.0 / f1;
      double di[3], dk[3];
      for (int c = 0; c < 3; c++) {
        di[c] = f1 * (d2[c] / (rij * rjk) - scp * d1[c] / r2ij);
        dk[c] = f1 * (d1[c] / (rij * rjk) - scp * d2[c] / r2jk);
      }
      atomic_add3(P.d, q.x, dv * di[0], dv * di[1], dv * di[2]);
      atomic_add3(P.d, q.z, dv * dk[0], dv * dk[1], dv * dk[2]);
      atomic_add3(P.d, q.y, -dv * (di[0] + dk[0]), -dv * (di[1] + dk[1]), -dv * (di[2] + dk[2]));
      rst_energy(P, s, S.S, q.w, e);
    }
  }
  for (int r = 0; r < S.nrw; r++) {
    int4 q = P.rw[S.rw_off + r];  // i, j, ih
    double4 prm = P.rw_p[S.rw_off + r];  // d, fk, aMorse, dMorse
    double e = 0;
    for (int i = q.x + threadIdx.x; i <= q.y; i += blockDim.x) {
      if (!((P.flags[i] & F_HEAVY) || q.z == 1)) continue;
      double3 xi = ld3(P.x, i);
      double dr[3] = {xi.x - S.xw[0], xi.y - S.xw[1], xi.z - S.xw[2]};
      double b = sqrt(dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2]);
      double db = b - prm.x, dv;
      if (db > 0.) { e += 0.5 * prm.y * db * db - prm.w; dv = prm.y * db / b; }
      else {
        double fexp = exp(prm.z * db);
        e += prm.w * (fexp * fexp - 2. * fexp);
        dv = -2. * prm.w * prm.z * (fexp - fexp * fexp) / b;
      }
      atomic_add3(P.d, i, dv * dr[0], dv * dr[1], dv * dr[2]);
    }
    double t = block_sum(e, sh);
    if (threadIdx.x == 0) atomicAdd(&P.E[s * QB_NE + QB_E_RST_PROTEIN], t);
    __syncthreads();
  }
}

// The solute force terms, one launch: blocks [0, pp) take nonbond_pp, then
// nonbond_qp, the bonded terms, nonbond_qq, the Q-atom bonded terms and the
// sequence/position/distance/angle/wall restraints, each on its own block
// range (blockIdx.y = system).  All of them add gradients with atomics, so
// they run concurrently.
struct SoluteGrid { int pp, qp, bonded, qq, qb, pre; };

template <int NSC>
__global__ void __launch_bounds__(256) k_solute_terms(DevPtrs P, SoluteGrid G) {
  int b = blockIdx.x;
  const int s = blockIdx.y;
  if (b < G.pp) { nb_pp_body(P, b, s, G.pp); return; }
  b -= G.pp;
  if (b < G.qp) { nb_qp_body<NSC>(P, b, s, G.qp); return; }
  b -= G.qp;
  if (b < G.bonded) { bonded_body(P, b, s, G.bonded); return; }
  b -= G.bonded;
  if (b < G.qq) { nb_qq_body(P, s); return; }
  b -= G.qq;
  if (b < G.qb) { qbonded_body(P, s); return; }
  b -= G.qb;
  if (b < G.pre) prestrain_body(P, s);
}

// watpol (md.f90:15122): water polarisation restraint, in two kernels.
// k_watpol_rank, one block per (shell, system): each member of the shell
// (angles and shells from k_pack_waters) is ranked by counting the members
// before it in (angle, water index) order, the reference's selection order
// with ties by water index.  The block also keeps
// the shell's running averages and updates theta_corr every 100 steps, in
// the reference's order (update first, then this step's average).
// k_watpol_force, one thread per water: target angle from the rank, restraint
// energy and the force on the water dipole.
constexpr int WPOL_BLOCK = 256;

__global__ void __launch_bounds__(WPOL_BLOCK) k_watpol_rank(DevPtrs P) {
  extern __shared__ unsigned char smem[];
  const int is = blockIdx.x, s = blockIdx.y;
  const SysDev &S = P.sys[s];
  if (!S.wpol || is >= S.nshell) return;
  const int nw = S.nwat;
  __shared__ int cnt;
  __shared__ double shsum[32];
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  const int8_t *wsh = P.wshell + S.woff;
  const double *wth = P.wtheta + S.woff;
  // member angles as bit patterns (non-negative doubles order like their bits)
  long long *kth = (long long *)smem;
  int *kiw = (int *)(kth + nw);                 // member water indices
  for (int w0 = 0; w0 < nw; w0 += WPOL_BLOCK) {
    const int iw = w0 + threadIdx.x;
    const bool mine = iw < nw && wsh[iw] == is;
    const unsigned bal = __ballot_sync(FULL, mine);
    int base = 0;
    if (lane == 0 && bal) base = atomicAdd(&cnt, __popc(bal));
    base = __shfl_sync(FULL, base, 0);
    if (mine) {
      const int k = base + __popc(bal & ((1u << lane) - 1u));
      kth[k] = __double_as_longlong(wth[iw]);
      kiw[k] = iw;
    }
  }
  __syncthreads();
  const int n = cnt;
  // rank = members before this one in (angle, water index) order; the
  // shared-memory reads are broadcasts
  double tsum = 0;
  for (int m = threadIdx.x; m < n; m += WPOL_BLOCK) {
    const long long th = kth[m];
    const int iw = kiw[m];
    // branch-free: both words of every key are read, no short-circuit
    int r[4] = {0, 0, 0, 0};
    int u = 0;
    for (; u + 4 <= n; u += 4) {
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const long long tu = kth[u + q];
        const int iu = kiw[u + q];
        r[q] += (int)(tu < th) + ((int)(tu == th) & (int)(iu < iw));
      }
    }
    for (; u < n; u++) {
      const long long tu = kth[u];
      const int iu = kiw[u];
      r[0] += (int)(tu < th) + ((int)(tu == th) & (int)(iu < iw));
    }
    P.wrank[S.woff + iw] = r[0] + r[1] + r[2] + r[3];
    tsum += __longlong_as_double(th);
  }
  double tot = block_sum(tsum, shsum);
  if (threadIdx.x == 0) {
    SysState &st = P.st[s];
    if (st.istep != 0 && st.istep % 100 == 0) {
      st.avtheta[is] = st.avtheta[is] / (float)100;
      st.avn_insh[is] = st.avn_insh[is] / (float)100;
      st.theta_corr[is] = st.theta_corr[is] + st.avtheta[is] - acosf(S.ws_cstb[is]);
      st.avtheta[is] = 0.0f;
      st.avn_insh[is] = 0.0f;
    }
    if (n > 0) {
      st.avtheta[is] = (float)((double)st.avtheta[is] + tot / (double)(float)n);
      st.avn_insh[is] = st.avn_insh[is] + (float)n;
    }
    P.wshn[s * MAX_SHELLS + is] = n;
  }
}

__global__ void __launch_bounds__(WPOL_BLOCK) k_watpol_force(DevPtrs P) {
  const int2 tile = P.wp_tiles[blockIdx.x];   // (system, first water)
  const int s = tile.x;
  const SysDev &S = P.sys[s];
  if (!S.wpol || S.nshell == 0) return;
  const int iw = tile.y + threadIdx.x;
  double epol = 0;
  const int is = iw < S.nwat ? (int)P.wshell[S.woff + iw] : -1;
  if (is >= 0) {
    const double pi = dev_pi();
    const SysState &st = P.st[s];
    const int n = P.wshn[s * MAX_SHELLS + is], rank = P.wrank[S.woff + iw];
    const double th = P.wtheta[S.woff + iw];
    const float tc = st.theta_corr[is];
    const float cstb = S.ws_cstb[is];
    float arg = 1.0f + (1.0f - 2.0f * (float)(rank + 1)) / (float)n;
    double th0 = (double)acosf(arg);
    th0 = th0 - 3. * sin(th0) * (double)cstb / 2.;
    if (th0 < 0.0) th0 = 0.0;
    if (th0 > pi) th0 = pi;
    double dth = th - th0 + (double)tc;
    epol = 0.5 * S.fkwpol * dth * dth;
    double dv = S.fkwpol * dth;
    int i = S.aoff + S.nsol + 3 * iw;
    double3 xO = ld3(P.x, i), x1 = ld3(P.x, i + 1), x2 = ld3(P.x, i + 2);
    double rmu[3] = {x1.x + x2.x - 2. * xO.x, x1.y + x2.y - 2. * xO.y, x1.z + x2.z - 2. * xO.z};
    double rm = sqrt(rmu[0] * rmu[0] + rmu[1] * rmu[1] + rmu[2] * rmu[2]);
    for (int c = 0; c < 3; c++) rmu[c] /= rm;
    double rcu[3] = {xO.x - S.xw[0], xO.y - S.xw[1], xO.z - S.xw[2]};
    double rc = sqrt(rcu[0] * rcu[0] + rcu[1] * rcu[1] + rcu[2] * rcu[2]);
    for (int c = 0; c < 3; c++) rcu[c] /= rc;
    double scp = rmu[0] * rcu[0] + rmu[1] * rcu[1] + rmu[2] * rcu[2];
    if (scp > 1.0) scp = 1.0;
    if (scp < -1.0) scp = -1.0;
    double f0 = sin(th);                 // th = acos(scp) of the same clamped scp
    if (fabs(f0) < 1.e-12) f0 = 1.e-12;
    f0 = -1.0 / f0;
    f0 = dv * f0;
    double gO[3], gH[3];
    for (int c = 0; c < 3; c++) {
      double f1 = (rcu[c] - rmu[c] * scp) / rm;
      double f2 = (rmu[c] - rcu[c] * scp) / rc;
      gO[c] = f0 * (-2. * f1 + f2);
      gH[c] = f0 * f1;
    }
    atomic_add3(P.d, i, gO[0], gO[1], gO[2]);
    atomic_add3(P.d, i + 1, gH[0], gH[1], gH[2]);
    atomic_add3(P.d, i + 2, gH[0], gH[1], gH[2]);
  }
  warp_add(&P.E[s * QB_NE + QB_E_RST_WATER_POL], epol);
}

// --------------------------------------------------------------- dynamics


// Leapfrog with Berendsen scaling (md.f90:4082-4110): one thread per atom.
// Kinetic energy of one atom into acc[4] (solute all, solute free, solvent
// all, solvent free), as temperature() sums it (md.f90:3817).
__device__ __forceinline__ void kin_add(const DevPtrs &P, const SysDev &S, int g, const double4 &v, double *acc) {
  double e = 0.5 * P.mass[g] * (v.x * v.x + v.y * v.y + v.z * v.z);
  bool free_ = !(P.flags[g] & F_EXCL);
  if (g - S.aoff < S.nsol) { acc[0] += e; if (free_) acc[1] += e; }
  else { acc[2] += e; if (free_) acc[3] += e; }
}

// Adds each lane's acc[4] to its system's kinetic-energy sums (s < 0: none):
// one warp reduction and one atomic per distinct system in the warp.  Every
// lane of the warp calls it.
__device__ __forceinline__ void kin_tally(DevPtrs &P, int s, const double *acc) {
  const int lane = threadIdx.x & 31;
  unsigned todo = __ballot_sync(FULL, s >= 0);
  while (todo) {
    const int leader = __ffs(todo) - 1;
    const int s0 = __shfl_sync(FULL, s, leader);
    const bool mine = s == s0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      double v = warp_sum(mine ? acc[k] : 0.0);
      if (lane == leader && v != 0.0) atomicAdd(&P.kin[s0 * 4 + k], v);
    }
    todo &= ~__ballot_sync(FULL, mine);
  }
}

// Leap-frog update (md.f90:4080-4108), one thread per atom of the list of
// atoms outside 3-constraint molecules: v from the gradient with the
// Berendsen factor of solute or solvent, x from v.  With SHAKE the reference
// then sets v = (x - xx)/dt for every atom (md.f90:4119); for atoms in no
// constraint that is done here (their x is final), for the others by the
// SHAKE kernels.  The kinetic energy of atoms whose velocity is final here
// is added to the system's sums.
__global__ void k_leapfrog(DevPtrs P) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int g = k < P.n_lf ? P.lf_atoms[k] : P.natoms_tot;   // the atoms outside 3-constraint molecules
  int s = -1;
  double acc[4] = {0, 0, 0, 0};
  // a system that raised an error stays where the failing step left it;
  // atoms of 3-constraint molecules are k_leapfrog_shake3's
  if (g < P.natoms_tot && P.st[P.asys[g]].frozen == 0 && !(P.flags[g] & F_SH3)) {
    s = P.asys[g];
    const SysDev &S = P.sys[s];
    double ts = (g - S.aoff) < S.nsol ? P.st[s].Tscale_sol : P.st[s].Tscale_solv;
    double w = (double)P.winv[g], dt = S.dt;
    double4 x = P.x[g], v = P.v[g], d = P.d[g];
    v.x = (v.x - d.x * w * dt) * ts;
    v.y = (v.y - d.y * w * dt) * ts;
    v.z = (v.z - d.z * w * dt) * ts;
    P.xx[g] = x;
    double4 xn = x;
    xn.x = x.x + v.x * dt;
    xn.y = x.y + v.y * dt;
    xn.z = x.z + v.z * dt;
    P.x[g] = xn;
    const bool shaken = P.flags[g] & F_SHAKE;
    if (S.has_shake && !shaken) {
      v.x = (xn.x - x.x) / dt;
      v.y = (xn.y - x.y) / dt;
      v.z = (xn.z - x.z) / dt;
    }
    P.v[g] = v;
    if (!shaken) kin_add(P, S, g, v, acc);
  }
  kin_tally(P, s, acc);
}


// Iteration counts of SHAKE molecules (the reference's niter, averaged per
// molecule) summed per system with the largest single count; every lane of
// the warp calls it (sys < 0 for lanes without a molecule).
__device__ __forceinline__ void shake_tally(DevPtrs &P, int sys, int its) {
  unsigned grp = __match_any_sync(FULL, sys);
  unsigned sum = __reduce_add_sync(grp, (unsigned)its);
  unsigned mx = __reduce_max_sync(grp, (unsigned)its);
  if (sys >= 0 && (threadIdx.x & 31) == __ffs(grp) - 1) {
    atomicAdd(&P.st[sys].shake_its, (unsigned long long)sum);
    atomicMax(&P.st[sys].shake_its_max, (int)mx);
  }
}

// One constraint update of shake (md.f90:14500-14540); true when the
// constraint was already within tolerance (it is still corrected, as there).
__device__ __forceinline__ bool shake_pair(double3 &xi, double3 &xj, const double3 &xxi, const double3 &xxj,
                                           float wi, float wj, double d2) {
  double xij[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
  double xij2 = xij[0] * xij[0] + xij[1] * xij[1] + xij[2] * xij[2];
  double diff = d2 - xij2;
  bool ready = fabs(diff) < 0.0001 * d2;
  double xxij[3] = {xxi.x - xxj.x, xxi.y - xxj.y, xxi.z - xxj.z};
  double scp = xij[0] * xxij[0] + xij[1] * xxij[1] + xij[2] * xxij[2];
  float wsum = wi + wj;
  double corr = diff / (2. * scp * (double)wsum);
  xi.x += xxij[0] * corr * (double)wi; xi.y += xxij[1] * corr * (double)wi; xi.z += xxij[2] * corr * (double)wi;
  xj.x -= xxij[0] * corr * (double)wj; xj.y -= xxij[1] * corr * (double)wj; xj.z -= xxij[2] * corr * (double)wj;
  return ready;
}

// shake (md.f90:14445) for molecules of three atoms and three constraints
// (rigid waters), one thread per molecule.  The atoms are relabelled on the
// host so that the constraints, in their own order, join (0,1), (0,2), (1,2);
// sweeps, readiness flags and the 1000-sweep limit are the reference's.
// k_leapfrog's update of atom g of system sys: the new velocity and position.
__device__ __forceinline__ void leapfrog_atom(const DevPtrs &P, int sys, int g, double4 &v, double3 &xn) {
  const SysDev &S = P.sys[sys];
  const double dt = S.dt;
  const double ts = (g - S.aoff) < S.nsol ? P.st[sys].Tscale_sol : P.st[sys].Tscale_solv;
  const double w = (double)P.winv[g];
  const double4 x = P.x[g], d = P.d[g];
  v = P.v[g];
  v.x = (v.x - d.x * w * dt) * ts;
  v.y = (v.y - d.y * w * dt) * ts;
  v.z = (v.z - d.z * w * dt) * ts;
  xn = make_double3(x.x + v.x * dt, x.y + v.y * dt, x.z + v.z * dt);
}

// Leapfrog (md.f90:4082-4110) and shake (14445) of one 3-constraint molecule
// per thread: the update of k_leapfrog for its three atoms, then the SHAKE
// sweeps on the new positions against the old ones, in registers; x and v
// are written once.  Without convergence the leapfrog values stay, as the
// separate kernels leave them (recomputed, bit for bit, on that rare path).
__global__ void __launch_bounds__(128, 6) k_leapfrog_shake3(DevPtrs P) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  int sys = -1, its = 0;
  double acc[4] = {0, 0, 0, 0};
  if (m < P.nsh3 && P.st[P.sh3_at[m].w].frozen == 0) {
    const int4 at = P.sh3_at[m];
    const double4 d2 = P.sh3_d2[m];
    sys = at.w;
    const int ids[3] = {at.x, at.y, at.z};
    double3 x0, x1, x2;
    {
      double4 v;
      leapfrog_atom(P, sys, at.x, v, x0);
      leapfrog_atom(P, sys, at.y, v, x1);
      leapfrog_atom(P, sys, at.z, v, x2);
    }
    const double3 r0 = ld3(P.x, at.x), r1 = ld3(P.x, at.y), r2 = ld3(P.x, at.z);
    const float w0 = P.winv[at.x], w1 = P.winv[at.y], w2 = P.winv[at.z];
    bool c0 = false, c1 = false, c2 = false;
    for (;;) {
      if (!c0) c0 = shake_pair(x0, x1, r0, r1, w0, w1, d2.x);
      if (!c1) c1 = shake_pair(x0, x2, r0, r2, w0, w2, d2.y);
      if (!c2) c2 = shake_pair(x1, x2, r1, r2, w1, w2, d2.z);
      its++;
      if (c0 && c1 && c2) break;
      if (its >= 1000) break;
    }
    if (c0 && c1 && c2) {
      const SysDev &S = P.sys[sys];
      const double dt = S.dt;
      double3 xs[3] = {x0, x1, x2}, rs[3] = {r0, r1, r2};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double4 o = P.x[ids[a]];
        o.x = xs[a].x; o.y = xs[a].y; o.z = xs[a].z;
        P.x[ids[a]] = o;
        double4 v = P.v[ids[a]];
        v.x = (xs[a].x - rs[a].x) / dt;
        v.y = (xs[a].y - rs[a].y) / dt;
        v.z = (xs[a].z - rs[a].z) / dt;
        P.v[ids[a]] = v;
        kin_add(P, S, ids[a], v, acc);
      }
    } else {
#pragma unroll
      for (int a = 0; a < 3; a++) {
        double4 v;
        double3 xn;
        leapfrog_atom(P, sys, ids[a], v, xn);
        double4 o = P.x[ids[a]];
        o.x = xn.x; o.y = xn.y; o.z = xn.z;
        P.x[ids[a]] = o;
        P.v[ids[a]] = v;
      }
      set_status(&P.st[sys], QB_ERR_SHAKE);
    }
  }
  shake_tally(P, sys, its);
  kin_tally(P, sys, acc);
}

// shake (md.f90:14445) for every other molecule, one block per molecule.
// The reference sweeps the constraints in order (Gauss-Seidel), skipping
// those already within tolerance.  The host groups them into levels: a
// constraint's level is one more than that of the latest earlier constraint
// sharing an atom, so constraints of one level touch disjoint atoms and every
// update they depend on comes from an earlier level.  Running the levels in
// order, each level in parallel, gives the reference's positions, readiness
// flags and sweep count exactly.  The molecule's atoms (position, winv) and
// its constraints (old bond vector, d2, readiness) live in shared memory, or
// in a per-molecule global scratch slice when they do not fit.
constexpr int SHG_BLOCK = 128;

__global__ void __launch_bounds__(SHG_BLOCK) k_shake_general(DevPtrs P) {
  extern __shared__ double4 shg_smem[];
  const int g = blockIdx.x;
  const int4 info = P.shg_info[g];       // atom offset, atoms, constraint offset, constraints
  const int4 info2 = P.shg_info2[g];     // level offset, levels, system, global scratch offset (-1: shared)
  const int na = info.y, nc = info.w, nlev = info2.y, sys = info2.z;
  double4 *ax = info2.w < 0 ? shg_smem : P.shg_scratch + info2.w;   // x, y, z, winv
  double4 *cx = ax + na;                                            // old bond vector, d2
  uint8_t *rdy = reinterpret_cast<uint8_t *>(cx + nc);
  const int *at = P.shg_at + info.x;
  const int2 *cij = P.shg_c + info.z;
  const int *lev = P.shg_lev + info2.x;
  // a system that raised an error stays where the failing step left it
  __shared__ int frozen;
  if (threadIdx.x == 0) frozen = P.st[sys].frozen;
  __syncthreads();
  if (frozen) return;
  for (int t = threadIdx.x; t < na; t += SHG_BLOCK) {
    double4 x = P.x[at[t]];
    x.w = (double)P.winv[at[t]];
    ax[t] = x;
  }
  for (int t = threadIdx.x; t < nc; t += SHG_BLOCK) {
    int2 ij = cij[t];
    double3 xi = ld3(P.xx, at[ij.x]), xj = ld3(P.xx, at[ij.y]);
    cx[t] = make_double4(xi.x - xj.x, xi.y - xj.y, xi.z - xj.z, P.shg_d2[info.z + t]);
    rdy[t] = 0;
  }
  __syncthreads();
  int its = 0;
  bool done = nc == 0;
  while (!done) {
    for (int L = 0; L < nlev; L++) {
      for (int t = lev[L] + threadIdx.x; t < lev[L + 1]; t += SHG_BLOCK) {
        if (rdy[t]) continue;
        const int2 ij = cij[t];
        const double4 c = cx[t];
        double4 xi = ax[ij.x], xj = ax[ij.y];
        double xij[3] = {xi.x - xj.x, xi.y - xj.y, xi.z - xj.z};
        double xij2 = xij[0] * xij[0] + xij[1] * xij[1] + xij[2] * xij[2];
        double diff = c.w - xij2;
        if (fabs(diff) < 0.0001 * c.w) rdy[t] = 1;
        double scp = xij[0] * c.x + xij[1] * c.y + xij[2] * c.z;
        float wi = (float)xi.w, wj = (float)xj.w;
        float wsum = wi + wj;
        double corr = diff / (2. * scp * (double)wsum);
        xi.x += c.x * corr * (double)wi; xi.y += c.y * corr * (double)wi; xi.z += c.z * corr * (double)wi;
        xj.x -= c.x * corr * (double)wj; xj.y -= c.y * corr * (double)wj; xj.z -= c.z * corr * (double)wj;
        ax[ij.x] = xi;
        ax[ij.y] = xj;
      }
      __syncthreads();
    }
    its++;
    bool mine = true;
    for (int t = threadIdx.x; t < nc; t += SHG_BLOCK) mine = mine && rdy[t];
    done = __syncthreads_and(mine);
    if (!done && its >= 1000) break;
  }
  double acc[4] = {0, 0, 0, 0};
  if (done) {
    const SysDev &S = P.sys[sys];
    for (int t = threadIdx.x; t < na; t += SHG_BLOCK) {
      const int g = at[t];
      double4 o = P.x[g];
      const double4 x = ax[t], xx = P.xx[g];
      o.x = x.x; o.y = x.y; o.z = x.z;
      P.x[g] = o;
      double4 v = P.v[g];
      v.x = (x.x - xx.x) / S.dt;
      v.y = (x.y - xx.y) / S.dt;
      v.z = (x.z - xx.z) / S.dt;
      P.v[g] = v;
      kin_add(P, S, g, v, acc);
    }
  } else if (threadIdx.x == 0) {
    set_status(&P.st[sys], QB_ERR_SHAKE);
  }
  __shared__ double ksh[32];
  for (int k = 0; k < 4; k++) {
    double t = block_sum(acc[k], ksh);
    if (threadIdx.x == 0 && t != 0.0) atomicAdd(&P.kin[sys * 4 + k], t);
  }
  if (threadIdx.x == 0) {
    atomicAdd(&P.st[sys].shake_its, (unsigned long long)its);
    atomicMax(&P.st[sys].shake_its_max, its);
  }
}

// Kinetic energy sums of the current velocities (the temperature before the
// first step, md.f90:3960): grid (blocks, systems).
constexpr int KIN_BLOCK = 256;

__global__ void __launch_bounds__(KIN_BLOCK) k_kinetic(DevPtrs P) {
  int s = blockIdx.y;
  const SysDev &S = P.sys[s];
  __shared__ double sh[32];
  double acc[4] = {0, 0, 0, 0};
  int il = blockIdx.x * KIN_BLOCK + threadIdx.x;
  if (il < S.natom) kin_add(P, S, S.aoff + il, P.v[S.aoff + il], acc);
  for (int k = 0; k < 4; k++) {
    double t = block_sum(acc[k], sh);
    if (threadIdx.x == 0 && t != 0.0) atomicAdd(&P.kin[s * 4 + k], t);
  }
}

// pot_energy's sums (md.f90:13500-13560): per-state Q totals, the
// lambda-weighted Q terms and the potential.  Lane st handles state st (its
// row loaded at once); lane 0 then adds the states in order and forms the
// totals from one load of the system's energy terms.
__device__ __forceinline__ void finalize_energy(DevPtrs &P, int s) {
  const SysDev &S = P.sys[s];
  const int lane = threadIdx.x;
  double *E = P.E + s * QB_NE;
  double w[7] = {0, 0, 0, 0, 0, 0, 0};   // this state's bond, angle, torsion, improper, qx_el, qx_vdw, restraint, x lambda
  if (lane < S.S) {
    double *q = P.EQ + ((size_t)s * MAXS + lane) * QB_NEQ;
    double r[QB_NEQ];
#pragma unroll
    for (int k = 0; k < QB_NEQ; k++) r[k] = q[k];
    const double lam = S.lambda[lane];
    r[QB_EQ_LAMBDA] = lam;
    r[QB_EQ_QX_EL] = r[QB_EQ_QQ_EL] + r[QB_EQ_QP_EL] + r[QB_EQ_QW_EL];
    r[QB_EQ_QX_VDW] = r[QB_EQ_QQ_VDW] + r[QB_EQ_QP_VDW] + r[QB_EQ_QW_VDW];
    r[QB_EQ_TOTAL] = r[QB_EQ_BOND] + r[QB_EQ_ANGLE] + r[QB_EQ_TORSION] + r[QB_EQ_IMPROPER] + r[QB_EQ_QX_EL] +
                     r[QB_EQ_QX_VDW] + r[QB_EQ_RESTRAINT];
    q[QB_EQ_LAMBDA] = r[QB_EQ_LAMBDA];
    q[QB_EQ_QX_EL] = r[QB_EQ_QX_EL];
    q[QB_EQ_QX_VDW] = r[QB_EQ_QX_VDW];
    q[QB_EQ_TOTAL] = r[QB_EQ_TOTAL];
    w[0] = r[QB_EQ_BOND] * lam; w[1] = r[QB_EQ_ANGLE] * lam; w[2] = r[QB_EQ_TORSION] * lam;
    w[3] = r[QB_EQ_IMPROPER] * lam; w[4] = r[QB_EQ_QX_EL] * lam; w[5] = r[QB_EQ_QX_VDW] * lam;
    w[6] = r[QB_EQ_RESTRAINT] * lam;
  }
  double e[QB_NE];
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < QB_NE; k++) e[k] = E[k];
  }
  for (int k = 0; k < S.S; k++) {
    double v[7];
#pragma unroll
    for (int c = 0; c < 7; c++) v[c] = __shfl_sync(FULL, w[c], k);
    if (lane == 0) {
      e[QB_E_Q_BOND] += v[0]; e[QB_E_Q_ANGLE] += v[1]; e[QB_E_Q_TORSION] += v[2]; e[QB_E_Q_IMPROPER] += v[3];
      e[QB_E_QX_EL] += v[4]; e[QB_E_QX_VDW] += v[5]; e[QB_E_RST_PROTEIN] += v[6];
    }
  }
  if (lane == 0) {
    e[QB_E_RST_TOTAL] = e[QB_E_RST_FIX] + e[QB_E_RST_SHELL] + e[QB_E_RST_PROTEIN] + e[QB_E_RST_SOLVENT_RADIAL] +
                        e[QB_E_RST_WATER_POL];
    e[QB_E_POTENTIAL] = e[QB_E_P_BOND] + e[QB_E_W_BOND] + e[QB_E_P_ANGLE] + e[QB_E_W_ANGLE] + e[QB_E_P_TORSION] +
                        e[QB_E_P_IMPROPER] + e[QB_E_PP_EL] + e[QB_E_PP_VDW] + e[QB_E_PW_EL] + e[QB_E_PW_VDW] +
                        e[QB_E_WW_EL] + e[QB_E_WW_VDW] + e[QB_E_Q_BOND] + e[QB_E_Q_ANGLE] + e[QB_E_Q_TORSION] +
                        e[QB_E_Q_IMPROPER] + e[QB_E_QX_EL] + e[QB_E_QX_VDW] + e[QB_E_RST_TOTAL] + e[QB_E_LRF];
    e[QB_E_KINETIC] = P.st[s].kinetic;
#pragma unroll
    for (int k = 0; k < QB_NE; k++) E[k] = e[k];
    if (!isfinite(e[QB_E_POTENTIAL])) set_status(&P.st[s], QB_ERR_NAN);
  }
  __syncwarp();
}

// End of a step, one warp per system.  mode 1 (a step): pot_energy's sums,
// then temperature (md.f90:3817) from the kinetic-energy sums of the
// leap-frog and SHAKE kernels, the Berendsen factors of the next step, the
// output and energy-file records of this step, and the step counter.
// mode 0: the temperature before the first step.  mode 2: the sums only
// (the energies after the loop).
__global__ void k_finish(DevPtrs P, int mode) {
  int s = blockIdx.x;
  const SysDev &S = P.sys[s];
  SysState &st = P.st[s];
  int lane = threadIdx.x;
  if (mode != 0) finalize_energy(P, s);
  if (mode == 2) return;
  if (mode == 1 && st.status != 0) {
    // failed at this step: no records, the step count stays at the failure,
    // and the kernels that move atoms skip the system from the next step on
    if (lane < 4) P.kin[s * 4 + lane] = 0.0;
    if (lane == 0) st.frozen = st.status;
    return;
  }
  if (lane == 0) {
    double tot[4];
    for (int k = 0; k < 4; k++) { tot[k] = P.kin[s * 4 + k]; P.kin[s * 4 + k] = 0.0; }
    const double kb = (double)kBoltzF;
    double Tfree_sol = tot[1], Tfree_solv = tot[3];
    double Tfree = Tfree_solv + Tfree_sol;
    double Temp = tot[0] + tot[2];
    st.kinetic = Temp;
    Temp = 2.0 * Temp / kb / (double)(float)S.Ndegf;
    Tfree = 2.0 * Tfree / kb / (double)(float)S.Ndegfree;
    if (S.detail_temps) {
      Tfree_sol = 2.0 * Tfree_sol / kb / (double)(float)S.Ndegfree_sol;
      Tfree_solv = 2.0 * Tfree_solv / kb / (double)(float)S.Ndegfree_solv;
    }
    double a = S.dt / S.tau_T;
    if (S.separate_scaling) {
      if (Tfree_solv != 0) st.Tscale_solv = S.Temp0 / Tfree_solv - 1.0;
      st.Tscale_solv = sqrt(1 + a * st.Tscale_solv);
      if (Tfree_sol != 0) st.Tscale_sol = S.Temp0 / Tfree_sol - 1.0;
      st.Tscale_sol = sqrt(1 + a * st.Tscale_sol);
    } else {
      if (Tfree != 0) st.Tscale_solv = S.Temp0 / Tfree - 1.0;
      st.Tscale_solv = sqrt(1 + a * st.Tscale_solv);
      st.Tscale_sol = st.Tscale_solv;
    }
    st.Temp = Temp;
    st.Tfree = Tfree;
    st.Tfree_sol = Tfree_sol;
    st.Tfree_solv = Tfree_solv;
    if (mode == 1) P.E[s * QB_NE + QB_E_KINETIC] = st.kinetic;
  }
  __syncwarp();
  if (mode == 1) {
    // output and energy-file records of this step, copied by the whole warp
    const int is = st.istep;
    const int rec_len = HIST_REC;
    for (int kind = 0; kind < 2; kind++) {
      int cyc = kind == 0 ? S.iout : S.iene;
      bool want = (is % cyc == 0) && (kind == 0 || is > 0);
      if (!want) continue;
      int c = st.hist_n[kind];
      const HistRef hr = *P.hr;
      if (c < hr.cap) {
        double *r = hr.hist + (((size_t)kind * P.nsys + s) * hr.cap + c) * rec_len;
        for (int k = lane; k < rec_len; k += 32)
          r[k] = k == 0 ? (double)is
                 : k <= QB_NE ? P.E[s * QB_NE + k - 1]
                 : k <= QB_NE + MAXS * QB_NEQ ? P.EQ[(size_t)s * MAXS * QB_NEQ + k - 1 - QB_NE]
                                              : P.offd_r[s * MAXS + k - 1 - QB_NE - MAXS * QB_NEQ];
      }
      __syncwarp();
      if (lane == 0) st.hist_n[kind] = c + 1;
    }
    __syncwarp();
    if (lane == 0) st.istep = is + 1;
  }
}

// ---------------------------------------------------------- periodic box

// put_back_in_box (md.f90:15477-15600), at the list steps of systems that put
// solute or solvent back: the box centre becomes the solute's mean position
// (all atoms without solute) unless it is rigid, then every molecule of the
// chosen range whose centre of mass lies beyond half an edge from the centre
// moves by one edge length along that axis.  Block per system; the centre is
// summed by one thread in the reference's atom order, molecules in parallel.
__global__ void k_put_back_in_box(DevPtrs P) {
  const int s = blockIdx.x;
  const SysDev &S = P.sys[s];
  SysState &st = P.st[s];
  if (!S.pbc || S.put_first >= S.put_last || (st.istep % S.NB) != 0) return;
  if (st.frozen) return;
  __shared__ double c[3];
  if (threadIdx.x == 0) {
    if (!S.rigid_center) {
      const int n = S.nsol > 0 ? S.nsol : S.natom;
      double b0 = 0, b1 = 0, b2 = 0;
      for (int i = 0; i < n; i++) {
        const double4 a = P.x[S.aoff + i];
        b0 += a.x; b1 += a.y; b2 += a.z;
      }
      st.boxc[0] = b0 / n; st.boxc[1] = b1 / n; st.boxc[2] = b2 / n;
    }
    for (int k = 0; k < 3; k++) c[k] = st.boxc[k];
  }
  __syncthreads();
  const double hi[3] = {c[0] + st.boxl[0] / 2, c[1] + st.boxl[1] / 2, c[2] + st.boxl[2] / 2};
  const double lo[3] = {c[0] - st.boxl[0] / 2, c[1] - st.boxl[1] / 2, c[2] - st.boxl[2] / 2};
  for (int m = S.put_first + threadIdx.x; m < S.put_last; m += blockDim.x) {
    const int a0 = P.mol_first[S.mol_off + m], a1 = P.mol_first[S.mol_off + m + 1];
    double cm[3] = {0, 0, 0};
    for (int j = a0; j < a1; j++) {
      const double4 a = P.x[j];
      const double w = P.mass_box[j];
      cm[0] += a.x * w; cm[1] += a.y * w; cm[2] += a.z * w;
    }
    const double mi = P.mol_minv[S.mol_off + m];
    double sh[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const double v = cm[k] * mi;
      sh[k] = v > hi[k] ? -st.boxl[k] : (v < lo[k] ? st.boxl[k] : 0.0);
    }
    if (sh[0] != 0.0 || sh[1] != 0.0 || sh[2] != 0.0)
      for (int j = a0; j < a1; j++) {
        double4 a = P.x[j];
        a.x += sh[0]; a.y += sh[1]; a.z += sh[2];
        P.x[j] = a;
      }
  }
}

// MC_volume's trial move (md.f90:15686-15722) for the systems in a volume
// move: every molecule's centre of mass scaled about the box centre by the
// ratio of new to old edge lengths, the molecule translated rigidly.  One
// thread per molecule.
__global__ void k_mc_scale(DevPtrs P) {
  const int s = blockIdx.y;
  const SysDev &S = P.sys[s];
  const SysState &st = P.st[s];
  if (!st.mc) return;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= S.nmol) return;
  const int a0 = P.mol_first[S.mol_off + m], a1 = P.mol_first[S.mol_off + m + 1];
  double cm[3] = {0, 0, 0};
  for (int j = a0; j < a1; j++) {
    const double4 a = P.x[j];
    const double w = P.mass_box[j];
    cm[0] += a.x * w; cm[1] += a.y * w; cm[2] += a.z * w;
  }
  const double mi = P.mol_minv[S.mol_off + m];
  double mv[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    cm[k] = cm[k] * mi;
    mv[k] = ((cm[k] - st.boxc[k]) * st.boxl[k] / st.mc_oldl[k] + st.boxc[k]) - cm[k];
  }
  for (int j = a0; j < a1; j++) {
    double4 a = P.x[j];
    a.x += mv[0]; a.y += mv[1]; a.z += mv[2];
    P.x[j] = a;
  }
}

}  // namespace qb
