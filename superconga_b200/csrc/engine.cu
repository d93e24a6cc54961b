// B200 engine of the SuperConga self-consistency hot path, behind the C ABI of
// include/scb200.h.
//
// One iteration (Context::compute, include/conga/Context.h:391-447) is a short
// sequence of launches on the context's stream:
//   accelerate        x <- F(x, g(x))                      (iterations >= 2)
//   extend_reference  order parameter extended past the grain (domain_ops.h),
//                     packed with A into one record per reference site
//   per angle chunk:
//     frame_fields    order parameter and Doppler shift along every column
//     sweep           gammaTilde down every trajectory column (stored), gamma up,
//                     Green sums over the Ozaki energies -> frame buffers;
//                     outgoing boundary values written in sparse order
//     halo            frame extension next to the boundary (domain_ops.h:11-69)
//     rotate_back     frame -> reference grid, accumulated angle by angle
//   finalize          Delta, j, free energy, residuals (ComputeOrderParameter.h,
//                     ComputeCurrent.h, ComputeFreeEnergy.h)
//   boundary          specular reflection through precomputed gather tables
//   poisson           the separable filters (ComputeVectorPotential.h) as one
//                     2D FFT convolution
// All static data (geometry in every frame, sparse indices, gather tables) is
// built once by setup.cpp and stays resident in HBM.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/scb200.h"
#include "device.cuh"
#include "setup.hpp"

using namespace scb;

namespace {

thread_local std::string g_create_error;

#define CUDA_TRY(expr)                                                          \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess)                                                      \
      throw EngineError(SC_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

struct EngineError {
  int code;
  std::string msg;
  EngineError(int c, std::string m) : code(c), msg(std::move(m)) {}
};

constexpr int REDUCE_THREADS = 256;
// Ozaki energies one sweep pass takes (the residues sit in shared memory);
// more are swept in passes of ENERGY_PASS (eight threads of four energies).
constexpr int SWEEP_MAX_ENERGIES = 64;
constexpr int ENERGY_PASS = 32;
constexpr int NQ = 48;  // partial-sum slots of the finalize reduction

// ------------------------------------------------------------------ kernels --

// The reference-grid fields the frame lookups gather, one record per site:
// rf[site * (nc + 1) + c] = (Re, Im) of order-parameter component c and
// rf[site * (nc + 1) + nc] = (A_x, A_y) of the induced vector potential, so
// that a bilinear corner costs one 16-byte load per field pair instead of two
// 8-byte loads from separate planes.  k_pack_reference copies the state
// (planar, [2 nc + 2][N0 * N0]) into it.
__global__ void k_pack_reference(int nc, int nn, const double *__restrict__ x, double2 *__restrict__ rf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nn) return;
  double2 *r = rf + (size_t)i * (nc + 1);
  for (int c = 0; c <= nc; ++c) r[c] = make_double2(x[(size_t)(2 * c) * nn + i], x[(size_t)(2 * c + 1) * nn + i]);
}

// FP32 copy of the records for the mixed-precision lookups (the FP32 sweep
// rounds the frame fields to FP32 anyway): half the bytes per gathered corner.
__global__ void k_round_reference(size_t n, const double2 *__restrict__ rf, float2 *__restrict__ rf32) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double2 v = rf[i];
  rf32[i] = make_float2((float)v.x, (float)v.y);
}

// Reference-grid extension of the order parameter (domain_ops.h:11-69):
// the order parameter everywhere, except label-0 sites next to the grain,
// which get the mean of their nearest grain sites; written into the records
// of k_pack_reference (field f = 2c + part of component c).
__global__ void k_extend_reference(int n_fields, int nn, int n_sites, int stride, const int *__restrict__ site,
                                   const int *__restrict__ off, const int *__restrict__ src,
                                   const double *__restrict__ in, double *__restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (k >= n_sites || f >= n_fields) return;
  const double *v = in + (size_t)f * nn;
  const int b = off[k], e = off[k + 1];
  double acc = v[src[b]];
  for (int i = b + 1; i < e; ++i) acc = __dadd_rn(acc, v[src[i]]);
  out[((size_t)site[k] * stride + (f >> 1)) * 2 + (f & 1)] = __ddiv_rn(acc, (double)(e - b));
}

// Element of the frame buffers: the per-angle Matsubara sums are accumulated in
// FP64 in the sweep and stored in the stepping precision (FP64 frames for the
// FP64 sweep; FP32 frames for the FP32 sweep, whose addends already carry the
// FP32 stepping error).  The angle sum in k_rotate_back is accumulated in FP64.
template <typename R>
struct FrameOf {
  using type = double2;
};
template <>
struct FrameOf<float> {
  using type = float2;
};
// LDOS frame element: FP64 in the plain form; FP32 in mixed precision, which
// holds the FP32 sweep's Im g exactly and halves the frame traffic.
template <typename R>
struct LdosOf {
  using type = double;
};
template <>
struct LdosOf<float> {
  using type = float;
};
template <typename F2>
__device__ __forceinline__ F2 frame_pair(double a, double b) {
  return F2{(decltype(F2::x))a, (decltype(F2::x))b};
}
__device__ __forceinline__ double2 as_d2(double2 v) { return v; }
__device__ __forceinline__ double2 as_d2(float2 v) { return make_double2(v.x, v.y); }

// Two consecutive double2 in one 256-bit load through the read-only path
// (ld.global.nc.v4.f64, sm_100); p must be 32-byte aligned.
__device__ __forceinline__ void ldg_d2x2(const double2 *p, double2 &a, double2 &b) {
  asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
      : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y)
      : "l"(p));
}

// A frame site's record is two frame elements, (Re F, Im F) then (Re g, Re I):
// 16 bytes in FP32, 32 in FP64, read with one load (the buffers are 256-byte
// aligned and the records packed).
struct FrameRec {
  double2 f, q;
};
__device__ __forceinline__ FrameRec load_rec(const float2 *fr, size_t i) {
  const float4 v = __ldg((const float4 *)fr + i);
  return FrameRec{make_double2(v.x, v.y), make_double2(v.z, v.w)};
}
__device__ __forceinline__ FrameRec load_rec(const double2 *fr, size_t i) {
  FrameRec r;
  ldg_d2x2(fr + 2 * i, r.f, r.q);
  return r;
}

template <typename R>
struct SweepArgs {
  int n0, n1, ne, nc, groups, log_groups, ept, n_items;
  int ne_stride;   // energies per boundary entry (all of them; ne counts this pass's)
  int accumulate;  // add the pass's Matsubara sums to the frame instead of storing them
  int burn_in, has_vp, has_ext, gauge;
  int slot_base;
  int pair;  // angle offset of the mirrored partner angle (n_angles / 2), 0 = unpaired
  int kmax;  // longest column of the chunk: rows of one scratch tile
  double h, lam_scale, flux_b, q, area;
  const int4 *items;  // (angle, x, first row, last row)
  const AngleParams *ang;
  const uint8_t *labels;
  const int *idx_in_g, *idx_out_g, *idx_in_gt, *idx_out_gt;
  const double *dist_in_g, *dist_out_g, *dist_in_gt, *dist_out_gt;
  const Cx<R> *bin_g, *bin_gt;
  Cx<R> *bout_g, *bout_gt;
  const double2 *rf;   // [n0*n0][nc + 1]: extended order parameter per component, then A (k_pack_reference)
  const float2 *rf32;  // the same records in FP32 (mixed precision: the FP32 sweep's lookups read these)
  const double *e_re, *e_im, *res;
  Cx<R> *scratch;   // [tile][row][energy][item of tile]
  R *scratch2;      // frame-field records [tile][row][item of tile] of (Re D, Im D, energy shift, label), in R
  typename FrameOf<R>::type *fr;  // frame records [slot][n1*n1][2]: (Re F, Im F), (Re g, Re I)
  typename LdosOf<R>::type *ldf;  // LDOS frame buffer [slot][n1*n1][energy]: Im g per real energy
};

// Scratch tiles: the items of one warp (32 / G trajectory columns, G = 2^lg
// threads per column) keep their sweep scratch together, row after row, so the
// rows a warp steps through are contiguous in memory instead of spread over
// planes the size of the chunk: gammaTilde [tile][row][energy][column of tile].
template <typename R>
__device__ __forceinline__ size_t scratch_index(const SweepArgs<R> &A, int lg, int item, int r, int e) {
  const int sh = 5 - lg;
  const size_t tile = (size_t)(item >> sh), k = (size_t)(item & ((1 << sh) - 1));
  return (((tile * A.kmax + r) * A.ne + e) << sh) + k;
}
// The packed FP32 sweep keeps energies 2p and 2p + 1 together as one 16-byte
// record (Re, Re, Im, Im): [tile][row][energy pair][column of tile], so a
// thread stores and loads both of its energies with one vector access.
template <typename R>
__device__ __forceinline__ size_t scratch_pair_index(const SweepArgs<R> &A, int lg, int item, int r, int p) {
  const int sh = 5 - lg;
  const size_t tile = (size_t)(item >> sh), k = (size_t)(item & ((1 << sh) - 1));
  return (((tile * A.kmax + r) * (size_t)((A.ne + 1) >> 1) + p) << sh) + k;
}
// Frame-field records, one per column site in the same tiles: (Re D, Im D,
// energy shift, frame label), [tile][row][column of tile], read by the sweep
// with one vector load per site.
template <typename R> struct Rec4;
template <> struct Rec4<double> { using type = double4; };
template <> struct Rec4<float> { using type = float4; };
template <typename R>
__device__ __forceinline__ size_t rec_index(const SweepArgs<R> &A, int lg, int item, int r) {
  const int sh = 5 - lg;
  const size_t tile = (size_t)(item >> sh), k = (size_t)(item & ((1 << sh) - 1));
  return ((tile * A.kmax + r) << sh) + k;
}

// Gauges, include/conga/riccati/energy_shift/Gauges.h:25-62.
__device__ __forceinline__ void gauge_potential(int gauge, double b, double area, double x,
                                                double y, double &ax, double &ay) {
  if (gauge == GAUGE_LANDAU) {
    ax = 0.0;
    ay = x * b;
  } else if (gauge == GAUGE_SYMMETRIC) {
    const double f = 0.5 * b;
    ax = -y * f;
    ay = x * f;
  } else {
    const double r2 = fmax(x * x + y * y, 1e-7);
    const double f = b * area / (2.0 * M_PI * r2);
    ax = -y * f;
    ay = x * f;
  }
}

// Reference records for the frame lookups: FP64 for the FP64 sweep, the FP32
// copy for the FP32 sweep.  ld_rec01 reads a site's component-0 and
// vector-potential records of a one-component grain in one load (32 or 16
// bytes).
__device__ __forceinline__ void ld_rec01(const SweepArgs<double> &A, size_t site, double2 &d, double2 &a) {
  ldg_d2x2(A.rf + site * 2, d, a);
}
__device__ __forceinline__ void ld_rec01(const SweepArgs<float> &A, size_t site, double2 &d, double2 &a) {
  const float4 v = __ldg((const float4 *)A.rf32 + site);
  d = make_double2(v.x, v.y);
  a = make_double2(v.z, v.w);
}
__device__ __forceinline__ double2 ld_rec(const SweepArgs<double> &A, size_t idx) { return __ldg(A.rf + idx); }
__device__ __forceinline__ double2 ld_rec(const SweepArgs<float> &A, size_t idx) {
  const float2 v = __ldg(A.rf32 + idx);
  return make_double2(v.x, v.y);
}

// Order parameter (OrderParameter::getRotatedGrid) and Doppler shift
// (computeEnergyShift, RiccatiSolver.h:127-176) at frame site (x, y).
template <typename R>
__device__ __forceinline__ void frame_fields(const SweepArgs<R> &A, const AngleParams &P, int x,
                                             int y, double &dre, double &dim, double &es) {
  const int n0 = A.n0;
  Bilinear b;
  dre = 0.0;
  dim = 0.0;
  const int st = A.nc + 1;
  // One component: a site's record (Delta, A) is 32 bytes, read with one
  // 256-bit load per corner, which also brings the corner's A when the
  // vector-potential lookup lands on the same corners (it differs only by the
  // rounding of its own rotation coefficients).
  const bool one = A.nc == 1;
  double2 ca[4];
  const bool inD = rotated_lookup(x, y, A.n1, n0, P.cD, P.sD, b);
  if (inD) {
    double c_re[4] = {0, 0, 0, 0}, c_im[4] = {0, 0, 0, 0};
    const int off[4] = {b.i00, b.i00 + 1, b.i00 + n0, b.i00 + n0 + 1};
    if (one) {
      const double et = P.eta[0];
      for (int k = 0; k < 4; ++k) {
        double2 v;
        ld_rec01(A, (size_t)off[k], v, ca[k]);
        c_re[k] += v.x * et;
        c_im[k] += v.y * et;
      }
    } else {
      for (int c = 0; c < A.nc; ++c) {
        const double et = P.eta[c];
        for (int k = 0; k < 4; ++k) {
          const double2 v = ld_rec(A, (size_t)off[k] * st + c);
          c_re[k] += v.x * et;
          c_im[k] += v.y * et;
        }
      }
    }
    dre = bilerp(c_re[0], c_re[1], c_re[2], c_re[3], b.xf, b.yf);
    dim = bilerp(c_im[0], c_im[1], c_im[2], c_im[3], b.xf, b.yf);
  }
  es = 0.0;
  if (A.has_vp || A.has_ext) {
    double ax = 0.0, ay = 0.0;
    const double off = -0.5 * (double)(A.n1 - 1);
    const double xp = ((double)x + off) * A.h, yp = ((double)y + off) * A.h;
    const double xr = xp * P.cE - yp * P.sE, yr = xp * P.sE + yp * P.cE;
    gauge_potential(A.gauge, A.flux_b, A.area, xr, yr, ax, ay);
    if (A.has_vp) {
      double rx = 0.0, ry = 0.0;
      Bilinear ba;
      if (rotated_lookup(x, y, A.n1, n0, P.cA, P.sA, ba)) {
        double2 v00, v01, v10, v11;
        if (one && inD && ba.i00 == b.i00) {
          v00 = ca[0];
          v01 = ca[1];
          v10 = ca[2];
          v11 = ca[3];
        } else {
          const size_t pa = (size_t)A.nc;
          v00 = ld_rec(A, pa + (size_t)ba.i00 * st);
          v01 = ld_rec(A, pa + (size_t)(ba.i00 + 1) * st);
          v10 = ld_rec(A, pa + (size_t)(ba.i00 + n0) * st);
          v11 = ld_rec(A, pa + (size_t)(ba.i00 + n0 + 1) * st);
        }
        rx = bilerp(v00.x, v01.x, v10.x, v11.x, ba.xf, ba.yf);
        ry = bilerp(v00.y, v01.y, v10.y, v11.y, ba.xf, ba.yf);
      }
      rx *= A.lam_scale;
      ry *= A.lam_scale;
      es = A.q * (P.vx * (rx + ax) + P.vy * (ry + ay));
    } else {
      es = A.q * (P.vx * ax + P.vy * ay);
    }
  }
}

__device__ __forceinline__ void group_sum(double &v, int groups, unsigned mask) {
  for (int o = groups >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o);
}

// Sum of four values over the G threads of a group, scattered: afterwards the
// thread whose group index has bits (b1 b0) in the two highest positions holds
// the total of value 2 b1 + b0 (G >= 4), or of values {2 b0, 2 b0 + 1} in v[0],
// v[1] (G = 2).  Halving the exchanged set in each of the first two rounds
// takes 3 (G = 2: 2, G = 8: 4) shuffles instead of 4 log2(G).
__device__ __forceinline__ void group_sum4_scatter(double v[4], int g, int log_groups, unsigned mask) {
  if (log_groups == 0) return;
  int o = 1 << (log_groups - 1);
  {  // keep two of four
    const bool up = (g & o) != 0;
    const double s0 = up ? v[0] : v[2], s1 = up ? v[1] : v[3];
    const double r0 = __shfl_xor_sync(mask, s0, o), r1 = __shfl_xor_sync(mask, s1, o);
    v[0] = (up ? v[2] : v[0]) + r0;
    v[1] = (up ? v[3] : v[1]) + r1;
  }
  o >>= 1;
  if (!o) return;
  {  // keep one of two
    const bool up = (g & o) != 0;
    const double sv = up ? v[0] : v[1];
    const double r = __shfl_xor_sync(mask, sv, o);
    v[0] = (up ? v[1] : v[0]) + r;
  }
  for (o >>= 1; o > 0; o >>= 1) v[0] += __shfl_xor_sync(mask, v[0], o);
}

// Rotated order parameter and Doppler shift of every site of every trajectory
// column of a chunk, written with the site's frame label as one record per
// site (rec_index) for the sweep.
// Block (FF_COLS, FF_ROWS): a warp covers 8 neighbouring columns x 4 rows, a
// compact patch of the frame whose rotated corners fall on few cache lines of
// the reference grid (a warp along one row touched ~20 sectors per gather).
constexpr int FF_COLS = 8, FF_ROWS = 16;
template <typename R>
__global__ void __launch_bounds__(FF_COLS * FF_ROWS) k_frame_fields(const SweepArgs<R> A, int rows_per_block) {
  const int item = blockIdx.x * FF_COLS + threadIdx.x;
  if (item >= A.n_items) return;
  const int4 it = A.items[item];
  const int a = it.x, x = it.y, lo = it.z, hi = it.w;
  const AngleParams &P = A.ang[a];  // read in place (a local copy went to the stack)
  const int r0 = blockIdx.y * rows_per_block;
  const int r1 = min(r0 + rows_per_block, hi - lo + 1);
  for (int r = r0 + threadIdx.y; r < r1; r += FF_ROWS) {
    double dre, dim, es;
    frame_fields(A, P, x, lo + r, dre, dim, es);
    const uint8_t lab = A.labels[(size_t)a * A.n1 * A.n1 + (size_t)(lo + r) * A.n1 + x];
    typedef typename Rec4<R>::type V4;
    ((V4 *)A.scratch2)[rec_index(A, A.log_groups, item, r)] = V4{(R)dre, (R)dim, (R)es, (R)lab};
  }
}

// One step of one coherence function at one site for EMAX interleaved
// energies (internal::computeStep, RiccatiSolverConfined.h:129-225): entry
// sites start from the stored boundary value with the partial step dist*h, grain
// sites take the midpoint step, exit sites also step on to the boundary and
// store the out-going value, sites outside the grain reset to zero.
template <typename R, int EMAX, bool KEL>
__device__ __forceinline__ void site_step(uint8_t l, uint8_t l_entry, uint8_t l_exit, R dre,
                                          R dim, R es, R pdre, R pdim, R pes, const R *ere,
                                          const R *eim, Cx<R> *coh, int ept, int ecount, R h,
                                          R dist_in, const Cx<R> *bin, R dist_out, Cx<R> *bout) {
  const bool entry = l == l_entry;
  const R sdre = entry ? dre : (dre + pdre) * R(0.5);
  const R sdim = entry ? dim : (dim + pdim) * R(0.5);
  const R ses = entry ? es : (es + pes) * R(0.5);
  const R st = entry ? dist_in * h : h;
#pragma unroll
  for (int j = 0; j < EMAX; ++j)
    if (j < ept) {
      Cx<R> g0 = coh[j];
      if (entry) g0 = (j < ecount) ? bin[j] : Cx<R>{R(0), R(0)};
      coh[j] = riccati_step<R>(sdre, sdim, KEL ? ses + ere[j] : ses, eim[j], g0, st);
    }
  if (l == l_exit) {
    const R sb = dist_out * h;
#pragma unroll
    for (int j = 0; j < EMAX; ++j)
      if (j < ept) {
        const Cx<R> bv = riccati_step<R>(dre, dim, KEL ? es + ere[j] : es, eim[j], coh[j], sb);
        if (j < ecount) bout[j] = bv;
      }
  }
  if (l == 0) {
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = Cx<R>{R(0), R(0)};
  }
}

// The step at a grain site (label 1) between two grain sites: midpoint fields,
// full step, no boundary bookkeeping (site_step handles the other labels).
template <typename R, int EMAX, bool KEL>
__device__ __forceinline__ void interior_step(R dre, R dim, R es, R pdre, R pdim, R pes,
                                              const R *ere, const R *eim, Cx<R> *coh, int ept,
                                              R h) {
  const R sdre = (dre + pdre) * R(0.5);
  const R sdim = (dim + pdim) * R(0.5);
  const R ses = (es + pes) * R(0.5);
#pragma unroll
  for (int j = 0; j < EMAX; ++j)
    if (j < ept) coh[j] = riccati_step<R>(sdre, sdim, KEL ? ses + ere[j] : ses, eim[j], coh[j], h);
}

// site_step and interior_step of the packed FP32 sweep: energies in pairs
// (riccati_step2), every thread with its full EMAX energies (the launch
// guarantees ept = EMAX).
// The real parts of energies j, j + 1 with the Doppler shift es added (KEL:
// real energies; Matsubara energies have none).
template <bool KEL>
__device__ __forceinline__ float2 ere_pair(const float *ere, int j, float es) {
  return KEL ? make_float2(es + ere[j], es + ere[j + 1]) : bc2(es);
}
template <int EMAX, bool KEL>
__device__ __forceinline__ void site_step_x2(uint8_t l, uint8_t l_entry, uint8_t l_exit, float dre, float dim,
                                             float es, float pdre, float pdim, float pes, const float *ere,
                                             const float *eim, Cx<float> *coh, int ept, int ecount, float h,
                                             float dist_in, const Cx<float> *bin, float dist_out,
                                             Cx<float> *bout) {
  const bool entry = l == l_entry;
  const float sdre = entry ? dre : (dre + pdre) * 0.5f;
  const float sdim = entry ? dim : (dim + pdim) * 0.5f;
  const float ses = entry ? es : (es + pes) * 0.5f;
  const float st = entry ? dist_in * h : h;
  const Cx<float> zero{0.0f, 0.0f};
#pragma unroll
  for (int j = 0; j < EMAX; j += 2) {
    if (j >= ept) break;
    Cx2 g0 = pack2(coh[j], coh[j + 1]);
    if (entry) g0 = pack2(j < ecount ? bin[j] : zero, j + 1 < ecount ? bin[j + 1] : zero);
    unpack2(riccati_step2(sdre, sdim, ere_pair<KEL>(ere, j, ses), make_float2(eim[j], eim[j + 1]), g0, st), coh[j],
            coh[j + 1]);
  }
  if (l == l_exit) {
    const float sb = dist_out * h;
#pragma unroll
    for (int j = 0; j < EMAX; j += 2) {
      if (j >= ept) break;
      Cx<float> b0, b1;
      unpack2(riccati_step2(dre, dim, ere_pair<KEL>(ere, j, es), make_float2(eim[j], eim[j + 1]),
                            pack2(coh[j], coh[j + 1]), sb),
              b0, b1);
      if (j < ecount) bout[j] = b0;
      if (j + 1 < ecount) bout[j + 1] = b1;
    }
  }
  if (l == 0) {
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = zero;
  }
}
template <int EMAX, bool KEL>
__device__ __forceinline__ void interior_step_x2(float dre, float dim, float es, float pdre, float pdim, float pes,
                                                 const float *ere, const float *eim, Cx<float> *coh, int ept,
                                                 float h) {
  const float sdre = (dre + pdre) * 0.5f;
  const float sdim = (dim + pdim) * 0.5f;
  const float ses = (es + pes) * 0.5f;
#pragma unroll
  for (int j = 0; j < EMAX; j += 2)
    if (j < ept)
      unpack2(riccati_step2(sdre, sdim, ere_pair<KEL>(ere, j, ses), make_float2(eim[j], eim[j + 1]),
                            pack2(coh[j], coh[j + 1]), h),
              coh[j], coh[j + 1]);
}

// Dispatch of one site's steps to the packed (PK) or the scalar form.
template <typename R, int EMAX, bool KEL, bool PK>
__device__ __forceinline__ void interior_any(R dre, R dim, R es, R pdre, R pdim, R pes, const R *ere,
                                             const R *eim, Cx<R> *coh, int ept, R h) {
  if constexpr (PK) interior_step_x2<EMAX, KEL>(dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, h);
  else interior_step<R, EMAX, KEL>(dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, h);
}
template <typename R, int EMAX, bool KEL, bool PK>
__device__ __forceinline__ void site_any(uint8_t l, uint8_t l_entry, uint8_t l_exit, R dre, R dim, R es, R pdre,
                                         R pdim, R pes, const R *ere, const R *eim, Cx<R> *coh, int ept,
                                         int ecount, R h, R dist_in, const Cx<R> *bin, R dist_out, Cx<R> *bout) {
  if constexpr (PK)
    site_step_x2<EMAX, KEL>(l, l_entry, l_exit, dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, ecount, h,
                            dist_in, bin, dist_out, bout);
  else
    site_step<R, EMAX, KEL>(l, l_entry, l_exit, dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, ecount, h,
                            dist_in, bin, dist_out, bout);
}

// The fused Riccati sweep of one chunk of angles.  G = 2^log_groups threads
// share one trajectory column (angle, x); thread g integrates Ozaki energies
// [g*ept, g*ept + ept).  gammaTilde runs down the column first and is kept in
// scratch; gamma then runs up and the Green sums over all energies are formed
// site by site (RiccatiSolverConfined.h:129-312, GreensFunctionStatic.h:92-157,
// ComputeFreeEnergy.h:106-160).  The frame order parameter and the energies come
// from scratch2; the coherence functions are integrated in R.
// KEL: real energies e_re + i e_im (the LDOS path, IntegrationIteratorKeldysh.h
// :219-389); instead of the energy sums, Im g of every energy is written to the
// LDOS frame buffer (GreensFunctionStatic.h:66-90, ComputeLDOS.h:123-144).
// One trajectory column (item) for thread g of its group; s_res holds the
// residues of the energies.
// STEP_PER_ANGLE: the Riccati step h/|v_F| is read per angle (a non-circular
// Fermi surface, and the batch); otherwise it is the uniform lattice spacing h
// of the circle, which stays a kernel parameter.
// Asynchronous global-to-shared copies of 16 bytes (cp.async.cg, through L2);
// with pred false nothing is read (the source must still be a valid address)
// and the 16 bytes are zero-filled.  Each thread waits only for its own
// copies (cp.async.wait_group), so no barrier is involved.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool pred) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(pred ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// The sweep's staging ring: every thread keeps the inputs of the next NS - 1
// sites of its column in flight (the site's frame-field record and, going up,
// the gammaTilde stored going down), copied asynchronously into shared memory
// ring[stage][16-byte unit][thread], so that the latency of these loads spans
// several sites' Riccati steps instead of one.  Used by the packed FP32 sweep
// with at most four energies per thread (128 threads per block; at most 40 KB
// of shared memory per block: 36 KB at four energies per thread, six stages).
// Measured on B200: C2 mixed sweep 5.69 -> 5.30 ms, C5 mixed LDOS sweep
// 79.5 -> 74.9 ms; the FP64 sweep, whose larger records leave room for three
// stages only, ran 2% (C2) to 18% (C5 LDOS) slower with it and keeps the
// one-site-ahead register prefetch.
template <typename R, int EMAX, bool PK>
struct SweepRing {
  static constexpr bool on = PK && EMAX <= 4;
  static constexpr int NV_REC = sizeof(R) == 8 ? 2 : 1;  // record: 32 or 16 bytes
  static constexpr int NV_GT = PK ? EMAX / 2 : EMAX;      // gammaTilde: one pair or one FP64 energy per unit
  static constexpr int NV = NV_REC + NV_GT;
  static constexpr int NS_FIT = (40 * 1024) / (NV * 128 * 16);
  static constexpr int NS = on ? (NS_FIT < 2 ? 2 : (NS_FIT > 8 ? 8 : NS_FIT)) : 1;
  static constexpr int NVD = on ? NV : 1;
};

// PK: the packed FP32 form (energies in pairs: riccati_step2, local_greens2 or
// greens_g_im2, the scratch in energy-pair records).  Each thread takes an
// even number of energies (the mapping's count rounded up, at most EMAX), so
// that every thread's first energy is even.
template <typename R, int EMAX, bool KEL, bool STEP_PER_ANGLE, int LG = -1, bool PK = false>
__device__ __forceinline__ void sweep_column(const SweepArgs<R> &A, const double *s_res, int item,
                                             int g, unsigned gmask) {
  static_assert(!PK || (std::is_same<R, float>::value && EMAX % 2 == 0), "packed sweep: FP32 pairs");
  const int lgc = LG >= 0 ? LG : A.log_groups;  // a compile-time group size when the launch knows it
  const int4 it = A.items[item];
  const int a = it.x, x = it.y, lo = it.z, hi = it.w;
  const int n1 = A.n1, ne = A.ne;
  const size_t nn1 = (size_t)n1 * n1;
  const size_t T = (size_t)(32 >> lgc);
  const R h = STEP_PER_ANGLE ? (R)A.ang[a].hs : (R)A.h;  // h / |v_F| of this angle
  // A compile-time group size comes with a full load (EMAX energies per
  // thread), a sweep that stores its frame sums, and no energy passes.
  const int ept = LG >= 0 ? EMAX : (PK ? ((A.ept + 1) & ~1) : A.ept);
  const bool burn_in = LG >= 0 ? false : A.burn_in != 0;
  const bool accumulate = LG >= 0 ? false : A.accumulate != 0;
  const int e0 = g * ept;
  int ecount = ne - e0;
  if (ecount > ept) ecount = ept;
  if (ecount < 0) ecount = 0;

  R eim[EMAX], ere[EMAX];
#pragma unroll
  for (int j = 0; j < EMAX; ++j) {
    eim[j] = (j < ecount) ? (R)A.e_im[e0 + j] : R(1);
    ere[j] = (KEL && j < ecount) ? (R)A.e_re[e0 + j] : R(0);
  }

  Cx<R> coh[EMAX];
  const size_t sb0 = PK ? scratch_pair_index(A, lgc, item, 0, e0 >> 1) : scratch_index(A, lgc, item, 0, e0);
  const size_t s_row = PK ? (size_t)((ne + 1) >> 1) * T : (size_t)ne * T;
  const size_t ax = (size_t)a * n1 + x;
  // Mirrored partner column (angle + pi, x -> n1 - 1 - x) when paired.
  const size_t pax = (size_t)(a + A.pair) * n1 + (n1 - 1 - x);
  // Without the staging ring, the next site's label, fields and stored
  // gammaTilde are loaded one site ahead so that their latency overlaps the
  // current site's Riccati steps.
  typedef typename Rec4<R>::type V4;
  using RG = SweepRing<R, EMAX, PK>;
  constexpr bool RING = RG::on;
  constexpr int NS = RG::NS;
  __shared__ float4 ring[NS][RG::NVD][128];
  const int tid = threadIdx.x;
  const int n_rows = hi - lo + 1;
  const V4 *fb = (const V4 *)A.scratch2 + rec_index(A, lgc, item, 0);
  // Copies of row `row` (record, and gammaTilde when with_gt) into the stage
  // of step `step`; one commit group per step, empty outside the column.
  auto ring_issue = [&](int step, int row, bool with_gt) {
    if constexpr (RING) {
      if (row >= 0 && row < n_rows) {
        const int sl = step % NS;
        const char *rp = (const char *)(fb + (size_t)row * T);
#pragma unroll
        for (int v = 0; v < RG::NV_REC; ++v) cp_async16(&ring[sl][v][tid], rp + 16 * v, true);
        if (with_gt) {
          if constexpr (PK) {
            const float4 *sc = (const float4 *)A.scratch + sb0 + (size_t)row * s_row;
#pragma unroll
            for (int jp = 0; jp < RG::NV_GT; ++jp) {
              const bool ok = 2 * jp < ecount;
              cp_async16(&ring[sl][RG::NV_REC + jp][tid], ok ? (const void *)(sc + (size_t)jp * T) : (const void *)rp,
                         ok);
            }
          } else {
            const Cx<R> *sc = A.scratch + sb0 + (size_t)row * s_row;
#pragma unroll
            for (int j = 0; j < RG::NV_GT; ++j) {
              const bool ok = j < ecount;
              cp_async16(&ring[sl][RG::NV_REC + j][tid], ok ? (const void *)(sc + (size_t)j * T) : (const void *)rp,
                         ok);
            }
          }
        }
      }
      cp_async_commit();
    }
  };
  auto ring_rec = [&](int step) -> V4 {
    const int sl = step % NS;
    if constexpr (sizeof(R) == 4) {
      const float4 v = ring[sl][0][tid];
      return V4{(R)v.x, (R)v.y, (R)v.z, (R)v.w};
    } else {
      const double2 u = *reinterpret_cast<const double2 *>(&ring[sl][0][tid]);
      const double2 w = *reinterpret_cast<const double2 *>(&ring[sl][RG::NV_REC - 1][tid]);
      return V4{(R)u.x, (R)u.y, (R)w.x, (R)w.y};
    }
  };
  auto ring_gt = [&](int step, Cx<R> *gt) {
    const int sl = step % NS;
    if constexpr (PK) {
#pragma unroll
      for (int jp = 0; jp < RG::NV_GT; ++jp) {
        const float4 v = ring[sl][RG::NV_REC + jp][tid];
        gt[2 * jp] = Cx<R>{(R)v.x, (R)v.z};
        gt[2 * jp + 1] = Cx<R>{(R)v.y, (R)v.w};
      }
    } else {
#pragma unroll
      for (int j = 0; j < RG::NV_GT; ++j) {
        const double2 v = *reinterpret_cast<const double2 *>(&ring[sl][RG::NV_REC + j][tid]);
        gt[j] = Cx<R>{(R)v.x, (R)v.y};
      }
    }
  };
  // ------------------------------------------------------ gammaTilde, down --
  {
    const int in_base = A.idx_in_gt[ax], out_base = A.idx_out_gt[ax];
    int nin = 0, nout = 0;
    R pdre = 0, pdim = 0, pes = 0;
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = Cx<R>{R(0), R(0)};
    V4 fr;
    if constexpr (RING) {
      for (int st = 0; st < NS - 1; ++st) ring_issue(st, n_rows - 1 - st, false);
    } else {
      fr = fb[(size_t)(hi - lo) * T];
    }
    for (int y = hi; y >= lo; --y) {
      const int r = y - lo;
      if constexpr (RING) {
        const int st = hi - y;
        ring_issue(st + NS - 1, r - (NS - 1), false);
        cp_async_wait<NS - 1>();
        fr = ring_rec(st);
      }
      const uint8_t l = (uint8_t)fr.w;
      // gammaTilde uses -conj(Delta) (RiccatiSolverConfined.h:74-79).
      const R dre = (R)(-fr.x), dim = (R)fr.y, es = (R)fr.z;
      if constexpr (!RING) {
        if (y > lo) fr = fb[(size_t)(r - 1) * T];
      }
      if (l == 1) {
        interior_any<R, EMAX, KEL, PK>(dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, h);
      } else {
        const bool entry = l == 3, exit = l == 2;
        const R din = entry ? (R)A.dist_in_gt[in_base + nin] : R(0);
        const R dout = exit ? (R)A.dist_out_gt[out_base + nout] : R(0);
        site_any<R, EMAX, KEL, PK>(l, 3, 2, dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, ecount, h,
                                   din, A.bin_gt + (size_t)(in_base + nin) * A.ne_stride + e0, dout,
                                   A.bout_gt + (size_t)(out_base + nout) * A.ne_stride + e0);
        if (A.pair && exit) {
          // gamma of the partner angle at its exit is conj(gammaTilde) here.
          const Cx<R> *src = A.bout_gt + (size_t)(out_base + nout) * A.ne_stride + e0;
          Cx<R> *dst = A.bout_g + (size_t)(A.idx_out_g[pax] + nout) * A.ne_stride + e0;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) dst[j] = Cx<R>{src[j].re, -src[j].im};
        }
        nin += entry;
        nout += exit;
      }
      if (!burn_in) {
        if constexpr (PK) {
          float4 *sc = (float4 *)A.scratch + sb0 + (size_t)r * s_row;
#pragma unroll
          for (int j = 0; j < EMAX; j += 2)
            if (j < ecount) sc[(size_t)(j >> 1) * T] = make_float4(coh[j].re, coh[j + 1].re, coh[j].im, coh[j + 1].im);
        } else {
          Cx<R> *sc = A.scratch + sb0 + (size_t)r * s_row;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) sc[(size_t)j * T] = coh[j];
        }
      }
      pdre = dre;
      pdim = dim;
      pes = es;
    }
    if constexpr (RING) cp_async_wait<0>();
  }
  // ----------------------------------------------------------- gamma, up --
  {
    const int in_base = A.idx_in_g[ax], out_base = A.idx_out_g[ax];
    int nin = 0, nout = 0;
    R pdre = 0, pdim = 0, pes = 0;
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = Cx<R>{R(0), R(0)};
    using Fr = typename FrameOf<R>::type;
    Fr *frs = A.fr + (size_t)(a - A.slot_base) * nn1 * 2;  // this angle's records
    // The value this thread stores when four or more threads share a column.
    auto *vdst = &frs->x + (lgc >= 2 ? (g >> (lgc - 2)) : 0);
    V4 fr;
    Cx<R> gt_nx[EMAX];
    // The stored gammaTilde of row r into gt_nx.
    auto load_gt = [&](int r) {
      if constexpr (PK) {
        const float4 *sc = (const float4 *)A.scratch + sb0 + (size_t)r * s_row;
#pragma unroll
        for (int j = 0; j < EMAX; j += 2)
          if (j < ecount) {
            const float4 v = sc[(size_t)(j >> 1) * T];
            gt_nx[j] = Cx<R>{v.x, v.z};
            gt_nx[j + 1] = Cx<R>{v.y, v.w};
          }
      } else {
        const Cx<R> *sc = A.scratch + sb0 + (size_t)r * s_row;
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) gt_nx[j] = sc[(size_t)j * T];
      }
    };
    if constexpr (RING) {
      for (int st = 0; st < NS - 1; ++st) ring_issue(st, st, !burn_in);
    } else {
      fr = fb[0];
      if (!burn_in) load_gt(0);
    }
    for (int y = lo; y <= hi; ++y) {
      const int r = y - lo;
      Cx<R> gt[EMAX];
      if constexpr (RING) {
        ring_issue(r + NS - 1, r + NS - 1, !burn_in);
        cp_async_wait<NS - 1>();
        fr = ring_rec(r);
        if (!burn_in) ring_gt(r, gt);
      }
      const uint8_t l = (uint8_t)fr.w;
      const R dre = (R)fr.x, dim = (R)fr.y, es = (R)fr.z;
      if constexpr (!RING) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j) gt[j] = gt_nx[j];
        if (y < hi) {
          fr = fb[(size_t)(r + 1) * T];
          if (!burn_in) load_gt(r + 1);
        }
      }
      if (l == 1) {
        interior_any<R, EMAX, KEL, PK>(dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, h);
      } else {
        const bool entry = l == 2, exit = l == 3;
        const R din = entry ? (R)A.dist_in_g[in_base + nin] : R(0);
        const R dout = exit ? (R)A.dist_out_g[out_base + nout] : R(0);
        site_any<R, EMAX, KEL, PK>(l, 2, 3, dre, dim, es, pdre, pdim, pes, ere, eim, coh, ept, ecount, h,
                                   din, A.bin_g + (size_t)(in_base + nin) * A.ne_stride + e0, dout,
                                   A.bout_g + (size_t)(out_base + nout) * A.ne_stride + e0);
        if (A.pair && exit) {
          // gammaTilde of the partner angle at its exit is conj(gamma) here.
          const Cx<R> *src = A.bout_g + (size_t)(out_base + nout) * A.ne_stride + e0;
          Cx<R> *dst = A.bout_gt + (size_t)(A.idx_out_gt[pax] + nout) * A.ne_stride + e0;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) dst[j] = Cx<R>{src[j].re, -src[j].im};
        }
        nin += entry;
        nout += exit;
      }
      pdre = dre;
      pdim = dim;
      pes = es;
      if (burn_in) continue;
      if constexpr (KEL) {
        if (l != 0) {
          typename LdosOf<R>::type *o = A.ldf + ((size_t)(a - A.slot_base) * nn1 + (size_t)y * n1 + x) * A.ne_stride + e0;
          if constexpr (PK) {
#pragma unroll
            for (int j = 0; j < EMAX; j += 2)
              if (j < ecount) {
                const float2 v = greens_g_im2(pack2(coh[j], coh[j + 1]), pack2(gt[j], gt[j + 1]));
                o[j] = v.x;
                if (j + 1 < ecount) o[j + 1] = v.y;
              }
          } else {
#pragma unroll
            for (int j = 0; j < EMAX; ++j)
              if (j < ecount) o[j] = greens_g_im<R>(coh[j], gt[j]);
          }
        }
        continue;
      }
      double sfr = 0.0, sfi = 0.0, sg = 0.0, si = 0.0;
      if constexpr (PK) {
        if (l != 0) {
          // Signs folded into the FP64 accumulation: sg = -sum r fre,
          // sfi = -sum r nfim, si = -sum r ni.
#pragma unroll
          for (int j = 0; j < EMAX; j += 2)
            if (j < ecount) {
              float2 fre, Fre, nfim, ni;
              local_greens2(pack2(coh[j], coh[j + 1]), pack2(gt[j], gt[j + 1]), dre, dim, fre, Fre, nfim, ni);
              const double r0 = s_res[e0 + j];
              sfr += r0 * (double)Fre.x;
              sfi -= r0 * (double)nfim.x;
              sg -= r0 * (double)fre.x;
              si -= r0 * (double)ni.x;
              if (j + 1 < ecount) {
                const double r1 = s_res[e0 + j + 1];
                sfr += r1 * (double)Fre.y;
                sfi -= r1 * (double)nfim.y;
                sg -= r1 * (double)fre.y;
                si -= r1 * (double)ni.y;
              }
            }
        }
      } else if (l != 0) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) {
            Cx<R> F;
            R gre, iim;
            local_greens<R>(coh[j], gt[j], dre, dim, F, gre, iim);
            const double rr = s_res[e0 + j];
            sfr += rr * (double)F.re;
            sfi += rr * (double)F.im;
            sg += rr * (double)gre;
            si += rr * (double)iim;
          }
      }
      // The mirrored partner angle is not stored: k_rotate_back reads it
      // from this frame at the mirrored site.
      const size_t fi = (size_t)y * n1 + x;
      double v[4] = {sfr, sfi, sg, -si};
      const int lg = lgc;
      group_sum4_scatter(v, g, lg, gmask);
      Fr *rec = frs + 2 * fi;
      if (lg == 0) {
        if (accumulate) {
          const double2 of = as_d2(rec[0]), og = as_d2(rec[1]);
          v[0] += of.x;
          v[1] += of.y;
          v[2] += og.x;
          v[3] += og.y;
        }
        rec[0] = frame_pair<Fr>(v[0], v[1]);
        rec[1] = frame_pair<Fr>(v[2], v[3]);
      } else if (lg == 1) {
        Fr *dst = rec + g;
        if (accumulate) {
          const double2 o = as_d2(*dst);
          v[0] += o.x;
          v[1] += o.y;
        }
        *dst = frame_pair<Fr>(v[0], v[1]);
      } else {
        const int sh = lg - 2;  // low bits below the two value bits
        if ((g & ((1 << sh) - 1)) == 0) {
          auto *dst = vdst + 4 * fi;
          if (accumulate) v[0] += (double)*dst;
          *dst = (decltype(Fr::x))v[0];
        }
      }
    }
    if constexpr (RING) cp_async_wait<0>();
  }
}

template <typename R, int EMAX, int MINB, bool KEL, bool STEP_PER_ANGLE = false, int LG = -1, bool PK = false>
__global__ void __launch_bounds__(128, MINB) k_sweep(const SweepArgs<R> A) {
  __shared__ double s_res[SWEEP_MAX_ENERGIES];  // residues of this pass's energies
  for (int e = threadIdx.x; e < A.ne && e < SWEEP_MAX_ENERGIES; e += blockDim.x) s_res[e] = A.res[e];
  __syncthreads();
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int lgk = LG >= 0 ? LG : A.log_groups, groups = 1 << lgk;
  const int item = tid >> lgk;
  const int g = tid & (groups - 1);
  const int lane = threadIdx.x & 31;
  const unsigned gmask = ((groups == 32) ? 0xffffffffu : ((1u << groups) - 1u)) << (lane & ~(groups - 1));
  if (item >= A.n_items) return;  // whole groups leave together (groups divide the warp)
  sweep_column<R, EMAX, KEL, STEP_PER_ANGLE, LG, PK>(A, s_res, item, g, gmask);
}

// The sweep of many grains in one persistent launch.  A work unit is one
// warp's worth of trajectory columns (32 / G of them) of one grain; warps take
// units from a global counter, longest columns first (the unit list is sorted
// by the host), so ragged grains share the GPU without a tail per grain.  All
// grain has its own G = 2^log_groups threads per column (the warp's unit
// belongs to one grain, so the mapping is uniform within a warp).
template <typename R, int EMAX, int MINB, bool PK = false>
__global__ void __launch_bounds__(128, MINB) k_sweep_batch(const SweepArgs<R> *__restrict__ args,
                                                           const int2 *__restrict__ units, int n_units,
                                                           int *counter) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int u = 0;
    if (lane == 0) u = atomicAdd(counter, 1);
    u = __shfl_sync(0xffffffffu, u, 0);
    if (u >= n_units) break;
    const int2 wu = units[u];
    const SweepArgs<R> &A = args[wu.x];
    const int lg = A.log_groups, groups = 1 << lg;
    const int g = lane & (groups - 1);
    const int sub = lane >> lg;
    const unsigned gmask = ((groups == 32) ? 0xffffffffu : ((1u << groups) - 1u)) << (lane & ~(groups - 1));
    const int item = wu.y + sub;
    if (item < A.n_items) sweep_column<R, EMAX, false, true, -1, PK>(A, A.res, item, g, gmask);
  }
}

// Frame extension next to the boundary for the angles of one chunk
// (ComputeOrderParameter.h:180-181, ComputeCurrent.h:149-150,
// ComputeFreeEnergy.h:265-266, all through domain_ops.h:11-69).
template <typename F2>
__global__ void k_halo(int n_entries, int entry0, int n1, const int *__restrict__ entry_angle,
                       int slot_base, const int *__restrict__ site, const int *__restrict__ off,
                       const int *__restrict__ src, F2 *fr) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_entries) return;
  const int e = entry0 + k;
  F2 *slot = fr + (size_t)(entry_angle[e] - slot_base) * n1 * n1 * 2;  // records of two F2
  const int b = off[e], en = off[e + 1];
  double2 f = as_d2(slot[2 * (size_t)src[b]]), q = as_d2(slot[2 * (size_t)src[b] + 1]);
  for (int i = b + 1; i < en; ++i) {
    const double2 f2 = as_d2(slot[2 * (size_t)src[i]]), q2 = as_d2(slot[2 * (size_t)src[i] + 1]);
    f.x = __dadd_rn(f.x, f2.x);
    f.y = __dadd_rn(f.y, f2.y);
    q.x = __dadd_rn(q.x, q2.x);
    q.y = __dadd_rn(q.y, q2.y);
  }
  const double cnt = (double)(en - b);
  slot[2 * (size_t)site[e]] = frame_pair<F2>(__ddiv_rn(f.x, cnt), __ddiv_rn(f.y, cnt));
  slot[2 * (size_t)site[e] + 1] = frame_pair<F2>(__ddiv_rn(q.x, cnt), __ddiv_rn(q.y, cnt));
}

// Rotation of the frame Green sums back to the reference grid, accumulated in
// angle order (ComputeOrderParameter.h:174-210, ComputeCurrent.h:142-173,
// ComputeFreeEnergy.h:260-279).
// With pair > 0 (mixed precision, mirrored angles) the frames hold only the
// angles [a_begin, a_end) of the first half; angle a + pair is read from the
// frame of a at the mirrored site (n1-1-x, n1-1-y) with gamma' = conj(gammaTilde),
// gammaTilde' = conj(gamma): F' = F, Re g' = -Re g, Re I' = Re I.  The angles
// are then accumulated in the order a, a + pair, a + 1, ...
// NC > 0 fixes the component count at compile time (the sums stay in
// registers); NC = 0 takes it from nc.  One component: four resident blocks
// per SM (64 registers) measured fastest on B200; more: three.
template <typename F2, int NC>
__global__ void __launch_bounds__(256, NC == 1 ? 4 : 3) k_rotate_back(int n0, int n1, int nc_, int a_begin,
                                                     int a_end, int pair, const AngleParams *__restrict__ ang,
                                                     const F2 *__restrict__ fr,
                                                     double *acc_d, double *acc_j, double *acc_fe) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= n0 || y >= n0) return;
  const size_t nn0 = (size_t)n0 * n0, nn1 = (size_t)n1 * n1;
  const size_t i = (size_t)y * n0 + x;
  const int nc = NC > 0 ? NC : nc_;
  double dr[NC > 0 ? NC : MAX_COMP], di[NC > 0 ? NC : MAX_COMP];
#pragma unroll
  for (int c = 0; c < nc; ++c) {
    dr[c] = acc_d[(size_t)(2 * c) * nn0 + i];
    di[c] = acc_d[(size_t)(2 * c + 1) * nn0 + i];
  }
  double jx = acc_j[i], jy = acc_j[nn0 + i], fe = acc_fe[i];
  const int last = (pair ? 2 : 1) * (a_end - a_begin);
  for (int k = 0; k < last; ++k) {
    const int a0 = a_begin + (pair ? k >> 1 : k);
    const bool mirrored = pair && (k & 1);
    const int a = mirrored ? a0 + pair : a0;
    const AngleParams &P = ang[a];
    // A site whose lookup falls outside the frame adds exact zeros (weights
    // 0, corners read at the frame origin): the same sums as skipping it, and
    // the loop stays free of branches so that the loads of consecutive angles
    // overlap.
    Bilinear b;
    const bool inside = rotated_lookup(x, y, n0, n1, P.cB, P.sB, b);
    if (!inside) b = Bilinear{0, 0.0, 0.0};
    const double pw = inside ? P.w : 0.0, psx = inside ? P.sx : 0.0, psy = inside ? P.sy : 0.0;
    FrameRec r00, r01, r10, r11;
    const size_t slot = (size_t)(a0 - a_begin) * nn1;
    if (!mirrored) {
      const size_t base = slot + b.i00;
      r00 = load_rec(fr, base); r01 = load_rec(fr, base + 1); r10 = load_rec(fr, base + n1); r11 = load_rec(fr, base + n1 + 1);
    } else {
      // corner (xi + dx, yi + dy) of angle a is site nn1 - 1 - i00 - dx - n1 dy of angle a0
      const size_t m = slot + (nn1 - 1 - (size_t)b.i00);
      r00 = load_rec(fr, m); r01 = load_rec(fr, m - 1); r10 = load_rec(fr, m - n1); r11 = load_rec(fr, m - n1 - 1);
    }
    const double fre = bilerp(r00.f.x, r01.f.x, r10.f.x, r11.f.x, b.xf, b.yf);
    const double fim = bilerp(r00.f.y, r01.f.y, r10.f.y, r11.f.y, b.xf, b.yf);
#pragma unroll
    for (int c = 0; c < nc; ++c) {
      const double et = P.eta[c];
      dr[c] += (fre * et) * pw;
      di[c] += (fim * et) * pw;
    }
    // Re g and Re I are interpolated once and weighted afterwards (the same
    // linear map as weighting the corners; the mirrored angle's Re g is minus
    // the stored one).
    const double gq = bilerp(r00.q.x, r01.q.x, r10.q.x, r11.q.x, b.xf, b.yf);
    const double g = mirrored ? -gq : gq;
    jx += g * psx;
    jy += g * psy;
    fe += bilerp(r00.q.y, r01.q.y, r10.q.y, r11.q.y, b.xf, b.yf) * pw;
  }
#pragma unroll
  for (int c = 0; c < nc; ++c) {
    acc_d[(size_t)(2 * c) * nn0 + i] = dr[c];
    acc_d[(size_t)(2 * c + 1) * nn0 + i] = di[c];
  }
  acc_j[i] = jx;
  acc_j[nn0 + i] = jy;
  acc_fe[i] = fe;
}

// LDOS frame extension next to the boundary, every energy of the block
// (ComputeLDOS.h:137-138 through domain_ops.h:11-69).
template <typename LF>
__global__ void k_halo_ldos(int n_entries, int entry0, int n1, int ne,
                            const int *__restrict__ entry_angle, int slot_base,
                            const int *__restrict__ site, const int *__restrict__ off,
                            const int *__restrict__ src, LF *ldf) {
  // one thread per (entry, energy), energy fastest: the LDOS frame is
  // [slot][site][energy]
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n_entries * ne) return;
  const int k = (int)(t / ne), en_ = (int)(t % ne);
  const int e = entry0 + k;
  LF *f = ldf + (size_t)(entry_angle[e] - slot_base) * n1 * n1 * ne + en_;
  const int b = off[e], en = off[e + 1];
  double v = f[(size_t)src[b] * ne];
  for (int i = b + 1; i < en; ++i) v = __dadd_rn(v, (double)f[(size_t)src[i] * ne]);
  f[(size_t)site[e] * ne] = (LF)__ddiv_rn(v, (double)(en - b));
}

// LDOS frames rotated back onto the reference grid and accumulated in angle
// order, Im part weighted by the integrand factor (ComputeLDOS.h:140-144,
// insertRotatedGridAdditive with Type::imag, GridFunctions_GPU.h:991-1054).
// The frame is energy-innermost ([slot][site][energy]): EL consecutive lanes
// take EL consecutive energies of one reference site, so that a warp's corner
// load reads whole runs of 32 / EL frame sites (two 128-byte lines for 32
// energies) instead of 32 scattered sites.  A block takes a TX x (256 / EL /
// TX) tile of reference sites; the bilinear lookups of its sites are computed
// once per angle into shared memory, RB_ANGLES angles at a time, and read
// back as broadcasts.  A site whose lookup falls outside the frame adds exact
// zeros (weight 0, corners read at the frame origin, which holds zeros): the
// same sums as skipping it, with a loop free of branches so that the loads of
// consecutive angles overlap.
constexpr int RB_ANGLES = 32;
template <int EL, int TX, typename LF>
__global__ void __launch_bounds__(256) k_rotate_back_ldos(int n0, int n1, int ne, int a_begin, int a_end,
                                                          const AngleParams *__restrict__ ang,
                                                          const LF *__restrict__ ldf, double *acc) {
  constexpr int SPB = 256 / EL, TY = SPB / TX;
  static_assert(SPB % TX == 0, "the site tile must fill the block");
  __shared__ int s_i00[RB_ANGLES][SPB];
  __shared__ double2 s_fxy[RB_ANGLES][SPB];
  __shared__ double s_w[RB_ANGLES][SPB];
  const int t = threadIdx.x;
  const int s = t / EL;
  const int x = blockIdx.x * TX + s % TX, y = blockIdx.y * TY + s / TX;
  const int e = blockIdx.z * EL + t % EL;
  const bool valid = x < n0 && y < n0 && e < ne;
  const size_t nn0 = (size_t)n0 * n0, nn1 = (size_t)n1 * n1;
  const size_t i = (size_t)y * n0 + x;
  const size_t dx = (size_t)ne, dy = (size_t)n1 * ne;
  double v = valid ? acc[(size_t)e * nn0 + i] : 0.0;
  for (int ab = a_begin; ab < a_end; ab += RB_ANGLES) {
    const int na = min(RB_ANGLES, a_end - ab);
    __syncthreads();  // every thread has read the previous angles' lookups
    for (int k = t; k < na * SPB; k += 256) {
      const int ka = k / SPB, ks = k % SPB;
      const int kx = blockIdx.x * TX + ks % TX, ky = blockIdx.y * TY + ks / TX;
      const AngleParams &P = ang[ab + ka];
      Bilinear b;
      const bool in = kx < n0 && ky < n0 && rotated_lookup(kx, ky, n0, n1, P.cB, P.sB, b);
      s_i00[ka][ks] = in ? b.i00 : 0;
      s_fxy[ka][ks] = in ? make_double2(b.xf, b.yf) : make_double2(0.0, 0.0);
      s_w[ka][ks] = in ? P.w : 0.0;
    }
    __syncthreads();
    if (!valid) continue;
    const LF *f = ldf + (size_t)(ab - a_begin) * nn1 * ne + e;
#pragma unroll 4
    for (int ka = 0; ka < na; ++ka) {
      const double2 fxy = s_fxy[ka][s];
      const double w = s_w[ka][s];
      const LF *c = f + (size_t)ka * nn1 * ne + (size_t)s_i00[ka][s] * ne;
      v += bilerp((double)c[0] * w, (double)c[dx] * w, (double)c[dy] * w, (double)c[dy + dx] * w, fxy.x, fxy.y);
    }
  }
  if (valid) acc[(size_t)e * nn0 + i] = v;
}

// ComputeLDOS::computePropertyFromGreens (ComputeLDOS.h:146-193): LDOS = -sum,
// zero outside the grain, residual against the block's previous LDOS, stored
// into the full LDOS array.
__global__ void __launch_bounds__(256) k_ldos_finalize(int n0, int n_fields, const uint8_t *__restrict__ dom,
                                                       const double *__restrict__ acc, double *ldos,
                                                       double *partial);

// Residual partial sums of one (old, new) pair: sum d^2, sum old^2, sum |d|,
// sum |old|, max |d|, max |old| (ComputeResidual.h:54-106).
struct Res6 {
  double s[6];
};
// Maximum that keeps a NaN (fmax drops it): a non-finite value anywhere in a
// residual reaches the residual, so a diverged state never reads as converged.
// Equal to fmax for numbers.
__device__ __forceinline__ double max_nan(double a, double b) {
  return (a != a) ? a : ((b != b) ? b : fmax(a, b));
}

__device__ __forceinline__ void res_add(double *q, double o, double n) {
  const double d = o - n;
  q[0] += d * d;
  q[1] += o * o;
  q[2] += fabs(d);
  q[3] += fabs(o);
  q[4] = max_nan(q[4], fabs(d));
  q[5] = max_nan(q[5], fabs(o));
}

// Block reduction of NQ slots: slots listed in max_mask are max-reduced.
__device__ void block_reduce(double *q, int nq, unsigned long long max_mask, double *out) {
  __shared__ double sh[REDUCE_THREADS];
  for (int k = 0; k < nq; ++k) {
    sh[threadIdx.x] = q[k];
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if ((int)threadIdx.x < s) {
        const double o = sh[threadIdx.x + s];
        sh[threadIdx.x] = ((max_mask >> k) & 1ull) ? max_nan(sh[threadIdx.x], o) : sh[threadIdx.x] + o;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) out[k] = sh[0];
    __syncthreads();
  }
}

// Slot layout of the finalize reduction.
//   [6c .. 6c+5]  order-parameter residual of component c (c < 4)
//   [24 .. 29]    current-density residual
//   30            sum of the free-energy kernel inside the grain
//   31 .. 34      sum |Delta_c|^2 inside the grain
//   35            sum B^2 over the lattice
//   36, 37        sum of the new current density (x, y)
constexpr unsigned long long FIN_MAX_MASK =
    (0x30ull) | (0x30ull << 6) | (0x30ull << 12) | (0x30ull << 18) | (0x30ull << 24);

// ComputeOrderParameter / ComputeCurrent / ComputeFreeEnergy
// ::computePropertyFromGreens, element-wise part and partial sums.
__global__ void __launch_bounds__(REDUCE_THREADS) k_finalize(
    int n0, int nc, double h, double jfactor, int has_vp, const uint8_t *__restrict__ dom,
    const double *__restrict__ coupling, const double *__restrict__ acc_d,
    const double *__restrict__ acc_j, const double *__restrict__ acc_fe,
    const double *__restrict__ delta, const double *__restrict__ avec, double *delta_new,
    double *j_real, double *partial) {
  const size_t nn = (size_t)n0 * n0;
  double q[NQ];
  for (int k = 0; k < NQ; ++k) q[k] = 0.0;
  const double inv_h = 1.0 / h;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    const bool in = dom[i] != 0;
    for (int c = 0; c < nc; ++c) {
      const double lc = coupling[c];
      for (int p = 0; p < 2; ++p) {
        const size_t k = (size_t)(2 * c + p) * nn + i;
        const double nv = in ? acc_d[k] * lc : 0.0;
        delta_new[k] = nv;
        res_add(&q[6 * c], delta[k], nv);
      }
      if (in) {
        const double o_re = delta[(size_t)(2 * c) * nn + i], o_im = delta[(size_t)(2 * c + 1) * nn + i];
        q[31 + c] += o_re * o_re + o_im * o_im;
      }
    }
    for (int d = 0; d < 2; ++d) {
      const size_t k = (size_t)d * nn + i;
      const double nv = in ? acc_j[k] * jfactor : 0.0;
      res_add(&q[24], j_real[k], nv);
      j_real[k] = nv;
      q[36 + d] += nv;
    }
    if (in) q[30] += acc_fe[i];
    if (has_vp) {
      // curl_kernel, GridFunctions_GPU.h:326-352.
      const int x = (int)(i % n0), y = (int)(i / n0);
      const int xn = min(x + 1, n0 - 1), xp = max(x - 1, 0);
      const int yn = min(y + 1, n0 - 1), yp = max(y - 1, 0);
      const double *ax = avec, *ay = avec + nn;
      const double dAydx = (ay[(size_t)y * n0 + xn] - ay[(size_t)y * n0 + xp]) / (double)(xn - xp);
      const double dAxdy = (ax[(size_t)yn * n0 + x] - ax[(size_t)yp * n0 + x]) / (double)(yn - yp);
      const double bz = (dAydx - dAxdy) * inv_h;
      q[35] += bz * bz;
    }
  }
  block_reduce(q, NQ, FIN_MAX_MASK, partial + (size_t)blockIdx.x * NQ);
}

__global__ void __launch_bounds__(256) k_ldos_finalize(int n0, int n_fields, const uint8_t *__restrict__ dom,
                                                       const double *__restrict__ acc, double *ldos,
                                                       double *partial) {
  double q[6] = {0, 0, 0, 0, 0, 0};
  const size_t nn = (size_t)n0 * n0, n = nn * n_fields;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const double nv = dom[i % nn] ? -acc[i] : 0.0;
    res_add(q, ldos[i], nv);
    ldos[i] = nv;
  }
  block_reduce(q, 6, 0x30ull, partial + (size_t)blockIdx.x * 6);
}

// Residual partials of a boundary gather (in-place update) or of any (old, new)
// pair of arrays.
__global__ void __launch_bounds__(REDUCE_THREADS) k_residual(size_t n, const double *__restrict__ o,
                                                             const double *__restrict__ nw,
                                                             double *partial) {
  double q[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    res_add(q, o[i], nw[i]);
  block_reduce(q, 6, 0x30ull, partial + (size_t)blockIdx.x * 6);
}

// Specular boundary condition through the precomputed gather table
// (BoundaryConditionSpecular.h:245-358): in[k] = sum_s w_s out[src_s] / wsum.
// The old value is read before it is replaced so the residual comes for free.
template <typename R>
__global__ void __launch_bounds__(REDUCE_THREADS) k_boundary(int n_in, int ne,
                                                             const int *__restrict__ src,
                                                             const double *__restrict__ w,
                                                             const double *__restrict__ wsum,
                                                             const Cx<R> *__restrict__ out,
                                                             Cx<R> *in, double *partial) {
  double q[6] = {0, 0, 0, 0, 0, 0};
  const size_t total = (size_t)n_in * ne;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(t / ne), e = (int)(t % ne);
    double re = 0.0, im = 0.0;
    for (int s = 0; s < 4; ++s) {
      const int sidx = src[4 * k + s];
      if (sidx < 0) continue;
      const Cx<R> v = out[(size_t)sidx * ne + e];
      const double ws = w[4 * k + s];
      re = __dadd_rn(re, __dmul_rn((double)v.re, ws));
      im = __dadd_rn(im, __dmul_rn((double)v.im, ws));
    }
    const double W = wsum[k];
    Cx<R> nv{R(0), R(0)};
    if (W > 0.0) nv = Cx<R>{(R)__ddiv_rn(re, W), (R)__ddiv_rn(im, W)};
    const Cx<R> ov = in[t];
    res_add(q, (double)ov.re, (double)nv.re);
    res_add(q, (double)ov.im, (double)nv.im);
    in[t] = nv;
  }
  block_reduce(q, 6, 0x30ull, partial + (size_t)blockIdx.x * 6);
}

// Initial boundary values: homogeneous solutions at every exit node
// (computeGammaFunctionInitialBoundaryTemplate_kernel,
// RiccatiSolverConfined.h:400-468).
template <typename R>
__global__ void k_boundary_initial(int n_out, int ne, int is_g, const int *__restrict__ node_a,
                                   const int *__restrict__ node_x, const int *__restrict__ node_y,
                                   SweepArgs<R> A, Cx<R> *bout) {
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (t >= (size_t)n_out * ne) return;
  const int k = (int)(t / ne), e = (int)(t % ne);
  const AngleParams P = A.ang[node_a[k]];
  double dre, dim, es;
  frame_fields(A, P, node_x[k], node_y[k], dre, dim, es);
  Cx<R> g, gt;
  riccati_homogeneous<R>((R)dre, (R)dim, (R)(es + A.e_re[e]), (R)A.e_im[e], g, gt);
  bout[t] = is_g ? g : gt;
}

// Subtracts the mean of each current component (ComputeVectorPotential.h:575-591).
__global__ void k_subtract_mean(int n0, const double *__restrict__ j, const double *__restrict__ scal,
                                int mean_slot, double *s) {
  const size_t nn = (size_t)n0 * n0;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= 2 * nn) return;
  const int d = (int)(i / nn);
  s[i] = j[i] - scal[mean_slot + d];
}

// ------------------------------------------------------- Poisson by FFT --
// The separable solve of ComputeVectorPotential::solve
// (ComputeVectorPotential.h:594-745) is A[r][c] = sum_{u,v} K(u, v) s[r+u][c+v]
// with s = j - <j> and the translation-invariant kernel
// K(u, v) = -h^2 scale * sum_k (+/-) f_k(u) f_k(v) built from the separable
// filters (ComputeVectorPotential.h:212-416).  It is evaluated as one linear
// convolution by zero-padded 2D FFTs of side P >= 2 N0 - 1 (P = 32 * 2^a 3^b 5^c):
// both current components travel in one complex array, s_x + i s_y, the
// kernel's spectrum is computed once at set-up.  O(P^2 log P) instead of
// O(K N0^3); the results agree with the direct filter sums to rounding.

// P-point FFT of every row in shared memory, P = 2^a 3^b 5^c <= 4096: the
// Stockham autosort formulation (Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC 2008) with mixed
// radices 2, 3, 4, 5, ping-ponging between two shared buffers.  Stage s with
// radix R and Ns = product of the earlier radices: butterfly j (< P/R) reads
// x[j + r P/R], twiddles it by w^(r k), k = j mod Ns, w = exp(-2 pi i / (Ns R)),
// takes the R-point DFT and writes y[(j / Ns) Ns R + k + r Ns].
// tw[q] = exp(-2 pi i q / P), q < P (conjugated for the inverse).
struct FftPlan {
  int n_stages;
  int radix[16];
};

__device__ __forceinline__ double2 cmul_d2(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// (x + i y) times s i, s = +1 or -1.
__device__ __forceinline__ double2 times_si(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// R-point DFTs with exponent sign s (-1 forward, +1 inverse); the constants
// are cos and sin of 2 pi / 3, 2 pi / 5 and 4 pi / 5.
template <int R>
__device__ __forceinline__ void dft_small(double2 *v, double s) {
  if constexpr (R == 2) {
    const double2 a = v[0], b = v[1];
    v[0] = make_double2(a.x + b.x, a.y + b.y);
    v[1] = make_double2(a.x - b.x, a.y - b.y);
  } else if constexpr (R == 4) {
    const double2 t0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
    const double2 t1 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
    const double2 t2 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
    const double2 t3 = times_si(make_double2(v[1].x - v[3].x, v[1].y - v[3].y), s);
    v[0] = make_double2(t0.x + t2.x, t0.y + t2.y);
    v[2] = make_double2(t0.x - t2.x, t0.y - t2.y);
    v[1] = make_double2(t1.x + t3.x, t1.y + t3.y);
    v[3] = make_double2(t1.x - t3.x, t1.y - t3.y);
  } else if constexpr (R == 3) {
    const double H3 = 0.86602540378443864676;  // sin(2 pi / 3) = sqrt(3) / 2
    const double2 t = make_double2(v[1].x + v[2].x, v[1].y + v[2].y);
    const double2 u = times_si(make_double2(H3 * (v[1].x - v[2].x), H3 * (v[1].y - v[2].y)), s);
    const double2 m = make_double2(v[0].x - 0.5 * t.x, v[0].y - 0.5 * t.y);
    v[0] = make_double2(v[0].x + t.x, v[0].y + t.y);
    v[1] = make_double2(m.x + u.x, m.y + u.y);
    v[2] = make_double2(m.x - u.x, m.y - u.y);
  } else {  // R == 5
    static_assert(R == 5, "radix 2, 3, 4 or 5");
    const double C1 = 0.30901699437494742410;   // cos(2 pi / 5) = (sqrt(5) - 1) / 4
    const double C2 = -0.80901699437494742410;  // cos(4 pi / 5) = -(sqrt(5) + 1) / 4
    const double S1 = 0.95105651629515357212;   // sin(2 pi / 5)
    const double S2 = 0.58778525229247312917;   // sin(4 pi / 5)
    const double2 a1 = make_double2(v[1].x + v[4].x, v[1].y + v[4].y);
    const double2 a2 = make_double2(v[2].x + v[3].x, v[2].y + v[3].y);
    const double2 b1 = make_double2(v[1].x - v[4].x, v[1].y - v[4].y);
    const double2 b2 = make_double2(v[2].x - v[3].x, v[2].y - v[3].y);
    const double2 p1 = make_double2(v[0].x + C1 * a1.x + C2 * a2.x, v[0].y + C1 * a1.y + C2 * a2.y);
    const double2 p2 = make_double2(v[0].x + C2 * a1.x + C1 * a2.x, v[0].y + C2 * a1.y + C1 * a2.y);
    const double2 q1 = times_si(make_double2(S1 * b1.x + S2 * b2.x, S1 * b1.y + S2 * b2.y), s);
    const double2 q2 = times_si(make_double2(S2 * b1.x - S1 * b2.x, S2 * b1.y - S1 * b2.y), s);
    v[0] = make_double2(v[0].x + a1.x + a2.x, v[0].y + a1.y + a2.y);
    v[1] = make_double2(p1.x + q1.x, p1.y + q1.y);
    v[4] = make_double2(p1.x - q1.x, p1.y - q1.y);
    v[2] = make_double2(p2.x + q2.x, p2.y + q2.y);
    v[3] = make_double2(p2.x - q2.x, p2.y - q2.y);
  }
}

// One Stockham stage of radix R (registers only: R is a template constant).
template <int R>
__device__ __forceinline__ void fft_stage(const double2 *a, double2 *b, int P, int ns,
                                          const double2 *__restrict__ tw, int inverse) {
  const int m = P / R, step = P / (ns * R);
  const double s = inverse ? 1.0 : -1.0;
  for (int j = threadIdx.x; j < m; j += blockDim.x) {
    const int k = j % ns;
    double2 v[R];
    v[0] = a[j];
#pragma unroll
    for (int r = 1; r < R; ++r) {
      double2 w = tw[r * k * step];
      if (inverse) w.y = -w.y;
      v[r] = cmul_d2(a[j + r * m], w);
    }
    dft_small<R>(v, s);
    const int d = (j / ns) * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) b[d + r * ns] = v[r];
  }
}

__global__ void __launch_bounds__(512) k_fft_rows(FftPlan plan, int P, const double2 *__restrict__ tw,
                                                  double2 *data, int inverse) {
  extern __shared__ double2 sm[];
  double2 *a = sm, *b = sm + P;
  double2 *row = data + (size_t)blockIdx.x * P;
  for (int i = threadIdx.x; i < P; i += blockDim.x) a[i] = row[i];
  __syncthreads();
  int ns = 1;
  for (int st = 0; st < plan.n_stages; ++st) {
    const int R = plan.radix[st];
    if (R == 4) fft_stage<4>(a, b, P, ns, tw, inverse);
    else if (R == 2) fft_stage<2>(a, b, P, ns, tw, inverse);
    else if (R == 3) fft_stage<3>(a, b, P, ns, tw, inverse);
    else fft_stage<5>(a, b, P, ns, tw, inverse);
    __syncthreads();
    double2 *t = a;
    a = b;
    b = t;
    ns *= R;
  }
  for (int i = threadIdx.x; i < P; i += blockDim.x) row[i] = a[i];
}

// out = transpose(in), P x P complex, 32 x 32 tiles.
__global__ void __launch_bounds__(256) k_fft_transpose(int P, const double2 *__restrict__ in, double2 *out) {
  __shared__ double2 tile[32][33];
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) tile[r][threadIdx.x] = in[(size_t)(y0 + r) * P + x0 + threadIdx.x];
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) out[(size_t)(x0 + r) * P + y0 + threadIdx.x] = tile[threadIdx.x][r];
}

// z[r][c] = s_x[r][c] + i s_y[r][c] inside the n x n lattice, 0 in the padding.
__global__ void k_fft_pack(int n, int P, const double *__restrict__ s, double2 *z) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)P * P) return;
  const int r = (int)(i / P), c = (int)(i % P);
  const size_t nn = (size_t)n * n;
  z[i] = (r < n && c < n) ? make_double2(s[(size_t)r * n + c], s[nn + (size_t)r * n + c]) : make_double2(0.0, 0.0);
}

__global__ void k_fft_mul(size_t count, const double2 *__restrict__ k, double2 *z) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double2 a = z[i], b = k[i];
  z[i] = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// a_x = Re z / P^2, a_y = Im z / P^2 on the n x n lattice.
__global__ void k_fft_unpack(int n, int P, double inv, const double2 *__restrict__ z, double *a) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t nn = (size_t)n * n;
  if (i >= nn) return;
  const int r = (int)(i / n), c = (int)(i % n);
  const double2 v = z[(size_t)r * P + c];
  a[i] = v.x * inv;
  a[nn + i] = v.y * inv;
}

// Scalars of one iteration, reduced from the block partials in a fixed order.
struct Scalars {
  double fe, fe_area, fe_mag, fe_mag_area;
  double res_op, res_j, res_fe, res_vp, res_bc, residual;
  double n_grain;
  double j_mean[2];
  double fe_area_prev;
  int first_j, first_fe;
  int conv_op, conv_j, conv_fe;
};

__device__ double residual_from(const double *t, size_t n_elem, int norm) {
  double numer, denom, eps = 1e-4;
  if (norm == NORM_L1) {
    numer = t[2];
    denom = t[3];
    eps *= (double)n_elem;
  } else if (norm == NORM_L2) {
    numer = sqrt(t[0]);
    denom = sqrt(t[1]);
    eps *= (double)n_elem;
  } else {
    numer = max_nan(t[4], 2.2250738585072014e-308);
    denom = max_nan(t[5], 2.2250738585072014e-308);
  }
  return numer / fmax(denom, eps);
}

// Sums (or maxima, for the slots set in max_mask) of nq slots over the
// nblocks rows of block partials: warp w reduces slots w, w + nwarps, ... in a
// fixed order (lane-strided, then a shuffle tree); results in t[0..nq).
__device__ void reduce_slots(const double *partial, int nblocks, int nq, unsigned long long max_mask,
                             double *t) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = w; k < nq; k += nw) {
    const bool mx = (max_mask >> k) & 1ull;
    double v = 0.0;
    for (int b = lane; b < nblocks; b += 32) {
      const double p = partial[(size_t)b * nq + k];
      v = mx ? max_nan(v, p) : v + p;
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double u = __shfl_xor_sync(0xffffffffu, v, o);
      v = mx ? max_nan(v, u) : v + u;
    }
    if (lane == 0) t[k] = v;
  }
  __syncthreads();
}

struct FinalizeConsts {
  int nc, norm, n_grain, has_vp;
  size_t n_elem_field;  // 2 * n0 * n0
  double temperature, h, lambda, conv, sum_inv;
  double log_t_tc[MAX_COMP];
};

// Free energy and the order-parameter / current residuals
// (ComputeFreeEnergy.h:281-414, ComputeOrderParameter.h:234-254,
// ComputeCurrent.h:184-211).
__global__ void k_scalars_a(FinalizeConsts C, const double *partial, int nblocks, Scalars *S) {
  __shared__ double t[NQ];
  reduce_slots(partial, nblocks, NQ, FIN_MAX_MASK, t);
  if (threadIdx.x != 0) return;
  double rop = 0.0;
  for (int c = 0; c < C.nc; ++c) rop = max_nan(rop, residual_from(&t[6 * c], C.n_elem_field, C.norm));
  S->res_op = rop;
  S->conv_op = rop < C.conv;
  const double rj = residual_from(&t[24], C.n_elem_field, C.norm);
  S->res_j = S->first_j ? C.conv * 0.1 : rj;
  S->conv_j = S->res_j < C.conv;
  S->first_j = 0;
  double nonmag = C.temperature * t[30];
  for (int c = 0; c < C.nc; ++c) nonmag += t[31 + c] * (C.log_t_tc[c] + C.sum_inv);
  double mag = 0.0;
  if (C.has_vp) mag += (0.5 / (C.lambda * C.lambda)) * t[35];
  const double la = C.h * C.h;
  const double fe_area = (nonmag + mag) / (double)C.n_grain;
  const double actual = fabs(S->fe_area_prev - fe_area) / fmax(fabs(S->fe_area_prev), 1e-4);
  S->res_fe = S->first_fe ? C.conv * 0.1 : actual;
  S->conv_fe = S->res_fe < C.conv;
  S->first_fe = 0;
  S->fe = (nonmag + mag) * la;
  S->fe_mag = mag * la;
  S->fe_area = fe_area;
  S->fe_mag_area = mag / (double)C.n_grain;
  S->fe_area_prev = fe_area;
  S->n_grain = (double)C.n_grain;
  S->j_mean[0] = t[36] / (double)C.n_grain;
  S->j_mean[1] = t[37] / (double)C.n_grain;
}

// Boundary and vector-potential residuals, total residual (Context.h:462-483).
__global__ void k_scalars_b(int norm, size_t n_elem_g, size_t n_elem_gt, size_t n_elem_vp,
                            int do_bc, int do_vp, int compute_mode, const double *p_bg, int nb_g,
                            const double *p_bgt, int nb_gt, const double *p_vp, int nb_vp, Scalars *S) {
  __shared__ double t[18];
  if (do_bc) {
    reduce_slots(p_bg, nb_g, 6, 0x30ull, &t[0]);
    reduce_slots(p_bgt, nb_gt, 6, 0x30ull, &t[6]);
  }
  if (do_vp) reduce_slots(p_vp, nb_vp, 6, 0x30ull, &t[12]);
  if (threadIdx.x != 0) return;
  if (do_bc) S->res_bc = max_nan(residual_from(&t[0], n_elem_g, norm), residual_from(&t[6], n_elem_gt, norm));
  if (do_vp) S->res_vp = residual_from(&t[12], n_elem_vp, norm);
  double r = S->res_vp;
  r = max_nan(S->res_bc, r);
  if (compute_mode) {
    r = max_nan(r, S->res_op);
    r = max_nan(r, S->res_j);
    r = max_nan(r, S->res_fe);
  }
  S->residual = r;
}

// ---------------------------------------------------------- accelerators --
// Per-field sums for CongAcc (CongAcc.h:371-385) and Barzilai-Borwein
// (BarzilaiBorwein.h:214-229): slots [3f] sum d^2, [3f+1] sum m^2, [3f+2] sum d m,
// where d = g - x and m is the running mean (CongAcc) or the previous d (BB).
__global__ void __launch_bounds__(REDUCE_THREADS) k_acc_sums(int nf, size_t nn, const double *__restrict__ x,
                                                             const double *__restrict__ gx,
                                                             const double *__restrict__ m,
                                                             double *partial) {
  const int f = blockIdx.y;
  double q[3] = {0, 0, 0};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nn;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t k = (size_t)f * nn + i;
    const double d = gx[k] - x[k], mv = m[k];
    q[0] += d * d;
    q[1] += mv * mv;
    q[2] += d * mv;
  }
  block_reduce(q, 3, 0, partial + ((size_t)f * gridDim.x + blockIdx.x) * 3);
}

constexpr int AND_MAX_RANK = 16;
struct AccState {
  double step[16];
  double inertia[16];
  double bb_step;
  int bb_iter;
  int initialized;
  // Anderson: iterations taken, the stored residuals' squared norms and
  // pairwise dot products (a stored pair does not change until its slot is
  // reused), and the weights of the current step.
  int and_iter;
  double and_sq[AND_MAX_RANK];
  double and_dot[AND_MAX_RANK][AND_MAX_RANK];
  double and_w[AND_MAX_RANK];
};

// Anderson::set (Anderson.h:267-289): the iterate and its residual
// d = g(x) - x go to slot iter mod rank (the oldest once all are used), and
// the block partials of |d|^2 and of d . D_j with the other stored residuals.
__global__ void __launch_bounds__(REDUCE_THREADS) k_and_store(size_t tot, int rank, const double *__restrict__ x,
                                                              const double *__restrict__ gx, double *hx,
                                                              double *hd, const AccState *st, double *partial) {
  const int it = st->and_iter, slot = it % rank, m = min(it + 1, rank);
  double q[AND_MAX_RANK];
  for (int j = 0; j < rank; ++j) q[j] = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < tot; k += (size_t)gridDim.x * blockDim.x) {
    const double d = gx[k] - x[k];
    hx[(size_t)slot * tot + k] = x[k];
    hd[(size_t)slot * tot + k] = d;
    for (int j = 0; j < m; ++j) q[j] += d * (j == slot ? d : hd[(size_t)j * tot + k]);
  }
  block_reduce(q, rank, 0, partial + (size_t)blockIdx.x * rank);
}

// Anderson::solve (Anderson.h:291-333): the bordered least-squares system
// [A 1; 1 0] [w; l] = [0; 1] with A_ij = D_i . D_j / mean |D|^2, solved by
// Gaussian elimination with partial pivoting; then the iteration count.
__global__ void k_and_solve(int rank, const double *partial, int nblocks, AccState *st) {
  __shared__ double t[AND_MAX_RANK];
  reduce_slots(partial, nblocks, rank, 0ull, t);
  if (threadIdx.x != 0) return;
  const int it = st->and_iter, slot = it % rank, m = min(it + 1, rank), mt = m + 1;
  for (int j = 0; j < m; ++j) {
    if (j == slot) continue;
    st->and_dot[slot][j] = t[j];
    st->and_dot[j][slot] = t[j];
  }
  st->and_sq[slot] = t[slot];
  double sr = 0.0;
  for (int i = 0; i < m; ++i) sr += st->and_sq[i];
  const double scale = 1.0 / (sr / (double)m);
  double M[AND_MAX_RANK + 1][AND_MAX_RANK + 1], rhs[AND_MAX_RANK + 1];
  for (int i = 0; i < mt; ++i) {
    rhs[i] = (i == mt - 1) ? 1.0 : 0.0;
    for (int j = 0; j < mt; ++j) M[i][j] = 1.0;
  }
  for (int i = 0; i < m; ++i) {
    M[i][i] = st->and_sq[i] * scale;
    for (int j = i + 1; j < m; ++j) {
      const double v = st->and_dot[i][j] * scale;
      M[i][j] = v;
      M[j][i] = v;
    }
  }
  M[mt - 1][mt - 1] = 0.0;
  for (int col = 0; col < mt; ++col) {
    int piv = col;
    for (int r = col + 1; r < mt; ++r)
      if (fabs(M[r][col]) > fabs(M[piv][col])) piv = r;
    if (piv != col) {
      for (int cc = 0; cc < mt; ++cc) {
        const double tmp = M[col][cc];
        M[col][cc] = M[piv][cc];
        M[piv][cc] = tmp;
      }
      const double tmp = rhs[col];
      rhs[col] = rhs[piv];
      rhs[piv] = tmp;
    }
    const double dg = M[col][col];
    for (int r = col + 1; r < mt; ++r) {
      const double f = M[r][col] / dg;
      for (int cc = col; cc < mt; ++cc) M[r][cc] -= f * M[col][cc];
      rhs[r] -= f * rhs[col];
    }
  }
  double w[AND_MAX_RANK + 1];
  for (int r = mt - 1; r >= 0; --r) {
    double v = rhs[r];
    for (int cc = r + 1; cc < mt; ++cc) v -= M[r][cc] * w[cc];
    w[r] = v / M[r][r];
  }
  for (int i = 0; i < AND_MAX_RANK; ++i) st->and_w[i] = i < m ? w[i] : 0.0;
  st->and_iter = it + 1;
}

// Anderson::computeInternal (Anderson.h:336-355): x = sum_i w_i (X_i + step D_i).
__global__ void k_and_update(size_t tot, int rank, double step, const double *__restrict__ hx,
                             const double *__restrict__ hd, const AccState *st, double *x) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= tot) return;
  const int m = min(st->and_iter, rank);  // already counts this iteration
  double v = 0.0;
  for (int i = 0; i < m; ++i) v += (hx[(size_t)i * tot + k] + hd[(size_t)i * tot + k] * step) * st->and_w[i];
  x[k] = v;
}

// CongAcc::computeInertia (CongAcc.h:300-356).
__device__ double congacc_inertia(double dn, double mn, double dot, double mincos) {
  double ea = dot / (dn * mn) - mincos, xa = 1.0;
  double eb = 1.0 - mincos, xb = 0.0;
  double x = 0.5 * (xa + xb);
  auto sgn = [](double v) { return (0.0 < v) - (v < 0.0); };
  for (int it = 0; it < 200; ++it) {
    const double y = 1.0 - x;
    const double numer = x * dot + y * dn * dn;
    const double denom = dn * sqrt(x * x * mn * mn + 2.0 * x * y * dot + y * y * dn * dn);
    const double err = numer / denom - mincos;
    const bool conv = fabs(err) < 0.01;
    if (sgn(err) == sgn(ea)) {
      ea = err;
      xa = x;
    } else {
      eb = err;
      xb = x;
    }
    if (sgn(ea) == sgn(eb)) break;
    x = 0.5 * (xa + xb);
    if (conv) break;
  }
  return x;
}

struct AccConsts {
  int kind, nf;
  double step_size, factor, mincos, smax, smin, drag;
};

// Scalar part of CongAcc::computeInternal (CongAcc.h:371-408) and
// BarzilaiBorwein::computeInternal (BarzilaiBorwein.h:211-232).
__global__ void k_acc_scalars(AccConsts C, const double *partial, int nblocks, AccState *st) {
  __shared__ double t[48];
  const int nf = C.nf;
  for (int f = 0; f < nf; ++f) reduce_slots(partial + (size_t)f * nblocks * 3, nblocks, 3, 0ull, &t[3 * f]);
  if (threadIdx.x != 0) return;
  if (!st->initialized) {
    for (int f = 0; f < nf; ++f) {
      st->step[f] = C.step_size;
      st->inertia[f] = 0.0;
    }
    st->bb_step = C.step_size;
    st->bb_iter = 0;
    st->initialized = 1;
  }
  if (C.kind == ACC_CONGACC) {
    for (int f = 0; f < nf; ++f) {
      const double d = sqrt(t[3 * f]), m = sqrt(t[3 * f + 1]);
      const double den = d * m;
      if (den > 0.0) {
        const double dot = t[3 * f + 2];
        const double cs = dot / den;
        st->step[f] *= pow(C.factor, cs);
        if (cs < C.mincos) st->inertia[f] = congacc_inertia(d, m, dot, C.mincos);
      }
      st->step[f] = fmin(fmax(st->step[f], C.smin), C.smax);
    }
  } else if (C.kind == ACC_BB) {
    if (st->bb_iter > 0) {
      // t: d^2 (= |d|^2), m^2 (= |dprev|^2), d.m (= d . dprev)
      double dd = 0.0, pp = 0.0, dp = 0.0;
      for (int f = 0; f < nf; ++f) {
        dd += t[3 * f];
        pp += t[3 * f + 1];
        dp += t[3 * f + 2];
      }
      const double dot = fabs(dp - pp);             // |dprev . (d - dprev)|
      const double ss = dd - 2.0 * dp + pp;         // |d - dprev|^2
      const double scale = (st->bb_iter % 2 == 0) ? dot / ss : pp / dot;
      st->bb_step *= scale;
    }
    st->bb_step = fmin(fmax(st->bb_step, C.smin), C.smax);
    st->bb_iter++;
  }
}

// Element-wise accelerator update: CongAcc (CongAcc.h:271-297), Picard
// (Picard.h:133-138), Polyak (Polyak.h:214-239), Barzilai-Borwein
// (BarzilaiBorwein.h:234-237).
__global__ void k_acc_update(AccConsts C, size_t nn, const double *__restrict__ gx, double *x,
                             double *m, const AccState *st) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)C.nf * nn) return;
  const int f = (int)(i / nn);
  const double d = gx[i] - x[i];
  if (C.kind == ACC_CONGACC) {
    const double in = st->inertia[f];
    const double mean = m[i] * in + d * (1.0 - in);
    m[i] = mean;
    x[i] += st->step[f] * mean;
  } else if (C.kind == ACC_PICARD) {
    x[i] += d * C.step_size;
  } else if (C.kind == ACC_POLYAK) {
    const double v = m[i] * (1.0 - C.drag) + d * C.step_size;
    m[i] = v;
    x[i] += v;
  } else {  // Barzilai-Borwein: m holds the previous difference
    m[i] = d;
    x[i] += d * st->bb_step;
  }
}

// Zero outside the reference domain (GeometryGroup::zeroValuesOutsideDomainRef).
__global__ void k_mask(int n_fields, size_t nn, const uint8_t *__restrict__ dom, double *v) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= (size_t)n_fields * nn) return;
  if (dom[i % nn] == 0) v[i] = 0.0;
}

template <typename R>
__global__ void k_to_interleaved(size_t n, const Cx<R> *__restrict__ in, double *out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[2 * i] = (double)in[i].re;
  out[2 * i + 1] = (double)in[i].im;
}
template <typename R>
__global__ void k_from_interleaved(size_t n, const double *__restrict__ in, Cx<R> *out) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = Cx<R>{(R)in[2 * i], (R)in[2 * i + 1]};
}

// FMA throughput probe: 8 independent FMA chains per thread, many warps.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, T a, T b, T *out) {
  T v[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) v[k] = (T)(threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = fma(v[k], a, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += v[k];
  if (s == (T)12345.678) out[0] = s;  // keeps the chains alive
}

// --------------------------------------------------------------- helpers --
template <typename T>
struct DevArray {
  T *p = nullptr;
  size_t n = 0;
  DevArray() = default;
  DevArray(const DevArray &) = delete;
  DevArray &operator=(const DevArray &) = delete;
  ~DevArray() { free(); }
  void alloc(size_t count) {
    free();
    n = count;
    if (count) CUDA_TRY(cudaMalloc(&p, count * sizeof(T)));
  }
  void upload(const std::vector<T> &v, cudaStream_t s) {
    alloc(v.size());
    if (n) CUDA_TRY(cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void zero(cudaStream_t s) {
    if (n) CUDA_TRY(cudaMemsetAsync(p, 0, n * sizeof(T), s));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

struct AdjBuffers;  // adjoint work buffers (adjoint.cuh)
struct AdjDeleter {
  void operator()(AdjBuffers *p) const;
};

struct Chunk {
  int a_begin, a_end;   // angles [a_begin, a_end)
  int item_begin, item_end;
  int kmax;             // longest column of the chunk
};

}  // namespace

// ------------------------------------------------------------------- context
struct sc_ctx {
  HostSetup S;
  int mode = SC_MODE_FP64;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the stream this context created
  std::string err;
  long long launches = 0;
  int device = 0;

  // static data
  DevArray<AngleParams> ang;
  DevArray<uint8_t> labels, dom;
  DevArray<int> idx_in_g, idx_out_g, idx_in_gt, idx_out_gt;
  DevArray<double> dist_in_g, dist_out_g, dist_in_gt, dist_out_gt;
  DevArray<int> bc_src_g, bc_src_gt;
  DevArray<double> bc_w_g, bc_w_gt, bc_ws_g, bc_ws_gt;
  DevArray<int> halo_site, halo_off, halo_src, halo_angle;
  DevArray<int> rext_site, rext_off, rext_src;
  DevArray<int4> items;
  DevArray<double> e_re, e_im, res, coupling;
  DevArray<double> filters;
  DevArray<int> filter_pos;
  DevArray<int> onode_a_g, onode_x_g, onode_y_g, onode_a_gt, onode_x_gt, onode_y_gt;
  std::vector<Chunk> chunks;
  int groups = 1, log_groups = 0, ept = 1;
  // Ozaki energies per sweep pass: all of them up to SWEEP_MAX_ENERGIES; above
  // that the sweep runs in passes of ENERGY_PASS energies that add into the
  // frame sums (low temperatures: T = 0.001 at cutoff 32 takes 281 energies).
  int e_pass = 1;
  bool emax2 = false;  // two-energies-per-thread sweep variant (tuning)
  int pair = 0;  // > 0: mixed mode sweeps angles [0, n/2) and mirrors them onto [n/2, n)

  // state: x = [delta | avec], g = [delta_new | a_new]
  DevArray<double> xstate, gstate, rfields, j_real;
  DevArray<double> rfields32;  // FP32 records (mixed precision), allocated as doubles
  std::vector<int4> h_items;  // trajectory columns (angle, x, first row, last row), host copy
  DevArray<double> acc_d, acc_j, acc_fe;
  DevArray<double> bnd;      // boundary storage (4 arrays), R-typed, viewed through pointers
  size_t bnd_off[4] = {0, 0, 0, 0};
  DevArray<double> scratch, scratch2, frames;
  DevArray<double> partial_fin, partial_bg, partial_bgt, partial_vp, partial_acc;
  DevArray<double> pois_s;
  // Poisson transform: side P = 32 * 2^a 3^b 5^c (radix plan), twiddles,
  // kernel spectrum, work arrays (complex).
  int fft_p = 0;
  FftPlan fft_plan{};
  DevArray<double> fft_tw, fft_kf, fft_z, fft_t;
  DevArray<double> acc_m;
  DevArray<double> and_x, and_d;  // Anderson history [rank][fields][N0*N0] (iterates, residuals)
  DevArray<AccState> acc_state;
  DevArray<Scalars> scalars;
  DevArray<double> tmp_io;
  int nb_fin = 0, nb_bnd = 0, nb_vp = 0, nb_acc = 0;

  // Work buffers of the sweep (scratch, fields, frame buffers): the
  // context's own arrays, or a batch's shared pool (batch_member).
  bool batch_member = false;
  // Frame buffers hold zeros wherever the sweep and the extension do not
  // write; with one chunk every slot always holds the same angle, so they are
  // cleared once instead of before every sweep.
  bool frames_zeroed = false;
  double *w_scratch = nullptr, *w_scratch2 = nullptr, *w_fr = nullptr;
  size_t need_scratch = 0, need_scratch2 = 0, need_frame = 0;  // bytes of each (frame: fg and gi each)

  std::unique_ptr<AdjBuffers, AdjDeleter> adj;  // allocated by the first sc_adjoint

  // LDOS postprocess: frame buffer, block accumulator, all energies.
  DevArray<double> ldf, ldos_acc, ldos_all;
  int ldos_block = -1;  // block whose energies the sweep uses

  bool boundary_initialized = false, first_compute = true;
  Scalars host_scalars{};

  // Optional CUDA-event timing of individual kernels (0 sweep, 1 rotate back,
  // 2 Poisson, 3 boundary condition), recorded on the launching stream.
  bool profiling = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof[5];

  // One steady-state iteration (accelerator step to scalars) captured as a
  // CUDA graph and replayed by sc_compute.  Every call that could change what
  // an iteration enqueues (state flags, field, stream, frame buffers) drops
  // it; sc_set_state only writes new values into the buffers the graph reads.
  cudaGraphExec_t iter_graph = nullptr;
  long long iter_graph_launches = 0;
  bool iter_graph_failed = false;
  void drop_graph() {
    if (iter_graph) cudaGraphExecDestroy(iter_graph);
    iter_graph = nullptr;
  }
  ~sc_ctx() { drop_graph(); }

  size_t nn0() const { return (size_t)S.n0 * S.n0; }
  size_t esize() const { return mode == SC_MODE_FP64 ? sizeof(Cx<double>) : sizeof(Cx<float>); }
  size_t ldos_esize() const { return mode == SC_MODE_FP64 ? sizeof(double) : sizeof(float); }
  // Bytes of one frame-buffer element (FrameOf<R>: float2 for the FP32 sweep).
  size_t frame_rec() const { return (mode == SC_MODE_MIXED && !S.keldysh) ? sizeof(float4) : 2 * sizeof(double2); }
  void *bnd_ptr(int which) const { return (char *)bnd.p + bnd_off[which]; }
  int n_bnd(int which) const {
    return which == 0 ? S.n_in_g : which == 1 ? S.n_out_g : which == 2 ? S.n_in_gt : S.n_out_gt;
  }
  bool has_vp() const { return S.lambda > 0.0; }
  int n_fields() const { return 2 * S.nc + (has_vp() ? 2 : 0); }
};

namespace {

struct ProfScope {
  sc_ctx *c;
  int k;
  cudaEvent_t e1 = nullptr;
  ProfScope(sc_ctx *ctx, int kernel) : c(ctx), k(kernel) {
    if (!c->profiling) return;
    cudaEvent_t e0;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, c->stream);
    c->prof[k].push_back({e0, e1});
  }
  ~ProfScope() {
    if (e1) cudaEventRecord(e1, c->stream);
  }
};

void check_launch(sc_ctx *c) {
  c->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) throw EngineError(SC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
}

unsigned grid1(size_t n, int threads) { return (unsigned)std::max<size_t>(1, (n + threads - 1) / threads); }

template <typename R>
SweepArgs<R> sweep_args(sc_ctx *c, const Chunk *ch, int burn_in) {
  const HostSetup &S = c->S;
  SweepArgs<R> A{};
  A.n0 = S.n0;
  A.n1 = S.n1;
  A.ne = S.ne;
  A.ne_stride = S.ne;
  A.nc = S.nc;
  A.groups = c->groups;
  A.log_groups = c->log_groups;
  A.ept = c->ept;
  A.n_items = ch ? ch->item_end - ch->item_begin : 0;
  A.burn_in = burn_in;
  A.has_vp = c->has_vp();
  A.flux_b = M_PI * S.flux_quanta / S.area;
  A.has_ext = std::fabs(A.flux_b) > 0.0;
  A.gauge = S.gauge;
  A.slot_base = ch ? ch->a_begin : 0;
  A.kmax = ch ? ch->kmax : 0;
  A.pair = (ch && ch->a_begin == 0 && ch->a_end == S.n_angles) ? c->pair : 0;
  A.h = S.h;
  A.lam_scale = c->has_vp() ? 1.0 / (S.lambda * S.lambda) : 0.0;
  A.q = (double)S.charge_sign;
  A.area = S.area;
  A.items = ch ? c->items.p + ch->item_begin : nullptr;
  A.ang = c->ang.p;
  A.labels = c->labels.p;
  A.idx_in_g = c->idx_in_g.p;
  A.idx_out_g = c->idx_out_g.p;
  A.idx_in_gt = c->idx_in_gt.p;
  A.idx_out_gt = c->idx_out_gt.p;
  A.dist_in_g = c->dist_in_g.p;
  A.dist_out_g = c->dist_out_g.p;
  A.dist_in_gt = c->dist_in_gt.p;
  A.dist_out_gt = c->dist_out_gt.p;
  A.bin_g = (const Cx<R> *)c->bnd_ptr(0);
  A.bout_g = (Cx<R> *)c->bnd_ptr(1);
  A.bin_gt = (const Cx<R> *)c->bnd_ptr(2);
  A.bout_gt = (Cx<R> *)c->bnd_ptr(3);
  A.rf = (const double2 *)c->rfields.p;
  A.rf32 = (const float2 *)c->rfields32.p;
  A.e_re = c->e_re.p;
  A.e_im = c->e_im.p;
  A.res = c->res.p;
  A.ldf = (typename LdosOf<R>::type *)c->ldf.p;
  A.scratch = (Cx<R> *)c->w_scratch;
  A.scratch2 = (R *)c->w_scratch2;
  A.fr = (typename FrameOf<R>::type *)c->w_fr;
  return A;
}

template <typename R>
void launch_frame_fields(sc_ctx *c, const Chunk &ch, const SweepArgs<R> &A) {
  if (!A.n_items) return;
  // Rows per block: a block's eight columns are walked down by its sixteen
  // row threads, so its gathers stay within a narrow strip of the reference
  // grid (L1 reuse) and each thread loads its column and angle once (C2:
  // 1024 rows per block 0.67 ms mixed, 1.47 ms FP64 against 0.86 and 1.90
  // with 64, and 1.24 / 2.88 with 16).
  const int rows = 64 * FF_ROWS;
  dim3 grid(grid1(A.n_items, FF_COLS), (unsigned)((ch.kmax + rows - 1) / rows));
  ProfScope prof(c, 4);
  k_frame_fields<R><<<grid, dim3(FF_COLS, FF_ROWS), 0, c->stream>>>(A, rows);
  check_launch(c);
}

template <typename R>
void launch_sweep_pass(sc_ctx *c, const SweepArgs<R> &A, unsigned blocks) {
  // Resident blocks per SM, fastest measured on B200 (606 x 606 d-wave square,
  // 256 angles, 14 energies, fixed-group kernels): FP64 three (four energies
  // per thread, 168 registers: 21.8 ms against 22.1 with four blocks and 24.4
  // with two); mixed in the packed FP32 form four (four energies per thread
  // in two pairs, four threads per column: 5.70 ms, 5.68 with three), or six
  // with two energies per thread.
  // The common mappings (four energies per thread and four threads per
  // column; mixed and LDOS: eight threads per column) are compiled with the
  // group size fixed, which turns the per-site group reduction, frame store
  // and tile addressing into straight-line code (C2: FP64 sweep -5%, mixed
  // -12%); other mappings take it at run time.
  static const char *minb_env = std::getenv("SCB_SWEEP_MINB");
  const int variant = minb_env ? std::atoi(minb_env) : (sizeof(R) == 8 ? 3 : (c->emax2 ? 6 : 1));
  const bool plain = !A.burn_in && !A.accumulate;  // what the fixed-group kernels assume
  if (c->S.fs_tight_binding) {
    // Non-circular Fermi surface: per-angle step, generic mappings.
    if (c->S.keldysh) {
      if (c->ept <= 4) k_sweep<R, 4, 1, true, true><<<blocks, 128, 0, c->stream>>>(A);
      else if (c->ept <= 8) k_sweep<R, 8, 1, true, true><<<blocks, 128, 0, c->stream>>>(A);
      else k_sweep<R, 16, 1, true, true><<<blocks, 128, 0, c->stream>>>(A);
    } else {
      if (c->ept <= 4) k_sweep<R, 4, 1, false, true><<<blocks, 128, 0, c->stream>>>(A);
      else if (c->ept <= 8) k_sweep<R, 8, 1, false, true><<<blocks, 128, 0, c->stream>>>(A);
      else k_sweep<R, 16, 1, false, true><<<blocks, 128, 0, c->stream>>>(A);
    }
  } else if (c->S.keldysh) {
    static const bool no_packed_kel = std::getenv("SCB_NO_PACKED") != nullptr;
    if constexpr (std::is_same<R, float>::value) {
      // Mixed-precision LDOS: four real energies per thread in two FP32 pairs.
      if (!no_packed_kel && c->ept == 4) {
        if (plain && c->log_groups == 3) k_sweep<R, 4, 1, true, false, 3, true><<<blocks, 128, 0, c->stream>>>(A);
        else k_sweep<R, 4, 1, true, false, -1, true><<<blocks, 128, 0, c->stream>>>(A);
        check_launch(c);
        return;
      }
    }
    if (plain && c->ept == 4 && c->log_groups == 3) k_sweep<R, 4, 1, true, false, 3><<<blocks, 128, 0, c->stream>>>(A);
    else if (c->ept <= 4) k_sweep<R, 4, 1, true><<<blocks, 128, 0, c->stream>>>(A);
    else if (c->ept <= 8) k_sweep<R, 8, 1, true><<<blocks, 128, 0, c->stream>>>(A);
    else k_sweep<R, 16, 1, true><<<blocks, 128, 0, c->stream>>>(A);
  } else if (c->ept <= 2 && c->emax2) {
    const bool g8 = plain && c->log_groups == 3 && c->ept == 2;
    if constexpr (std::is_same<R, float>::value) {
      // Two energies per thread: the packed FP32 form (both energies in one
      // FFMA2 / FMUL2 / FADD2 per operation).
      static const bool no_packed = std::getenv("SCB_NO_PACKED") != nullptr;
      if (!no_packed && c->ept == 2 && (variant >= 6 || variant == 4)) {
        if (variant >= 6 && g8) k_sweep<R, 2, 6, false, false, 3, true><<<blocks, 128, 0, c->stream>>>(A);
        else if (variant >= 6) k_sweep<R, 2, 6, false, false, -1, true><<<blocks, 128, 0, c->stream>>>(A);
        else if (g8) k_sweep<R, 2, 4, false, false, 3, true><<<blocks, 128, 0, c->stream>>>(A);
        else k_sweep<R, 2, 4, false, false, -1, true><<<blocks, 128, 0, c->stream>>>(A);
        check_launch(c);
        return;
      }
    }
    if (variant >= 6 && g8) k_sweep<R, 2, 6, false, false, 3><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant >= 6) k_sweep<R, 2, 6, false><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 4 && g8) k_sweep<R, 2, 4, false, false, 3><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 5 && g8) k_sweep<R, 2, 5, false, false, 3><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 5) k_sweep<R, 2, 5, false><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 3) k_sweep<R, 2, 3, false><<<blocks, 128, 0, c->stream>>>(A);
    else k_sweep<R, 2, 4, false><<<blocks, 128, 0, c->stream>>>(A);
  } else if (c->ept <= 4) {
    if constexpr (std::is_same<R, float>::value) {
      // Four energies per thread in mixed precision (energy passes of low
      // temperatures, or a mapping chosen by SCB_ENERGY_GROUPS): two FP32 pairs.
      static const bool no_packed4 = std::getenv("SCB_NO_PACKED") != nullptr;
      if (!no_packed4 && c->ept == 4) {
        const bool g4 = plain && c->log_groups == 2;
        if (variant == 3 && g4) k_sweep<R, 4, 3, false, false, 2, true><<<blocks, 128, 0, c->stream>>>(A);
        else if (variant == 3) k_sweep<R, 4, 3, false, false, -1, true><<<blocks, 128, 0, c->stream>>>(A);
        else if (g4) k_sweep<R, 4, 4, false, false, 2, true><<<blocks, 128, 0, c->stream>>>(A);
        else k_sweep<R, 4, 4, false, false, -1, true><<<blocks, 128, 0, c->stream>>>(A);
        check_launch(c);
        return;
      }
    }
    if (variant == 4 && plain && c->log_groups == 2 && c->ept == 4) k_sweep<R, 4, 4, false, false, 2><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 4) k_sweep<R, 4, 4, false><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 5) k_sweep<R, 4, 5, false><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 3 && plain && c->log_groups == 2 && c->ept == 4) k_sweep<R, 4, 3, false, false, 2><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 2 && plain && c->log_groups == 2 && c->ept == 4) k_sweep<R, 4, 2, false, false, 2><<<blocks, 128, 0, c->stream>>>(A);
    else if (variant == 3) k_sweep<R, 4, 3, false><<<blocks, 128, 0, c->stream>>>(A);
    else k_sweep<R, 4, 1, false><<<blocks, 128, 0, c->stream>>>(A);
  } else if (c->ept <= 8) {
    k_sweep<R, 8, 1, false><<<blocks, 128, 0, c->stream>>>(A);
  } else {
    k_sweep<R, 16, 1, false><<<blocks, 128, 0, c->stream>>>(A);
  }
  check_launch(c);
}

template <typename R>
void launch_sweep(sc_ctx *c, const Chunk &ch, int burn_in) {
  SweepArgs<R> A = sweep_args<R>(c, &ch, burn_in);
  const size_t threads = (size_t)A.n_items * c->groups;
  if (!threads) return;
  const unsigned blocks = grid1(threads, 128);
  launch_frame_fields<R>(c, ch, A);
  ProfScope prof(c, 0);
  const int ne = c->S.ne, pass = c->e_pass;
  if (pass >= ne) {
    launch_sweep_pass<R>(c, A, blocks);
    return;
  }
  // Energy passes: each pass steps energies [e, e + pass) of every column
  // from their own boundary values and adds its Matsubara sums to the frame.
  for (int e = 0; e < ne; e += pass) {
    SweepArgs<R> P = A;
    P.ne = std::min(pass, ne - e);
    P.accumulate = e > 0;
    P.e_re += e;
    P.e_im += e;
    P.res += e;
    P.bin_g += e;
    P.bout_g += e;
    P.bin_gt += e;
    P.bout_gt += e;
    P.ldf += e;  // LDOS frames: energy-innermost, this pass's slice
    launch_sweep_pass<R>(c, P, blocks);
  }
}

void extend_reference(sc_ctx *c) {
  const HostSetup &S = c->S;
  const int nn = (int)c->nn0();
  k_pack_reference<<<grid1(nn, 256), 256, 0, c->stream>>>(S.nc, nn, c->xstate.p, (double2 *)c->rfields.p);
  check_launch(c);
  const int ns = (int)S.rext_site.size();
  if (ns) {
    dim3 grid(grid1(ns, 128), 2 * S.nc);
    k_extend_reference<<<grid, 128, 0, c->stream>>>(2 * S.nc, nn, ns, S.nc + 1, c->rext_site.p, c->rext_off.p,
                                                    c->rext_src.p, c->xstate.p, c->rfields.p);
    check_launch(c);
  }
  if (c->rfields32.p) {
    const size_t n = (size_t)(S.nc + 1) * nn;
    k_round_reference<<<grid1(n, 256), 256, 0, c->stream>>>(n, (const double2 *)c->rfields.p,
                                                           (float2 *)c->rfields32.p);
    check_launch(c);
  }
}

template <typename R>
void boundary_condition(sc_ctx *c) {
  const HostSetup &S = c->S;
  ProfScope prof(c, 3);
  k_boundary<R><<<c->nb_bnd, REDUCE_THREADS, 0, c->stream>>>(
      S.n_in_g, S.ne, c->bc_src_g.p, c->bc_w_g.p, c->bc_ws_g.p, (const Cx<R> *)c->bnd_ptr(1),
      (Cx<R> *)c->bnd_ptr(0), c->partial_bg.p);
  check_launch(c);
  k_boundary<R><<<c->nb_bnd, REDUCE_THREADS, 0, c->stream>>>(
      S.n_in_gt, S.ne, c->bc_src_gt.p, c->bc_w_gt.p, c->bc_ws_gt.p, (const Cx<R> *)c->bnd_ptr(3),
      (Cx<R> *)c->bnd_ptr(2), c->partial_bgt.p);
  check_launch(c);
}

template <typename R>
void boundary_initial(sc_ctx *c) {
  const HostSetup &S = c->S;
  extend_reference(c);
  SweepArgs<R> A = sweep_args<R>(c, nullptr, 1);
  const size_t ng = (size_t)S.n_out_g * S.ne, ngt = (size_t)S.n_out_gt * S.ne;
  if (ng) {
    k_boundary_initial<R><<<grid1(ng, 128), 128, 0, c->stream>>>(
        S.n_out_g, S.ne, 1, c->onode_a_g.p, c->onode_x_g.p, c->onode_y_g.p, A, (Cx<R> *)c->bnd_ptr(1));
    check_launch(c);
  }
  if (ngt) {
    k_boundary_initial<R><<<grid1(ngt, 128), 128, 0, c->stream>>>(
        S.n_out_gt, S.ne, 0, c->onode_a_gt.p, c->onode_x_gt.p, c->onode_y_gt.p, A,
        (Cx<R> *)c->bnd_ptr(3));
    check_launch(c);
  }
  boundary_condition<R>(c);
  c->boundary_initialized = true;
}

void launch_scalars_b(sc_ctx *c, int do_bc, int do_vp, int compute_mode, size_t n_elem_vp = 0) {
  const HostSetup &S = c->S;
  if (!n_elem_vp) n_elem_vp = 2 * c->nn0();
  k_scalars_b<<<1, 256, 0, c->stream>>>(S.norm, (size_t)2 * S.n_in_g * S.ne,
                                         (size_t)2 * S.n_in_gt * S.ne, n_elem_vp, do_bc, do_vp,
                                         compute_mode, c->partial_bg.p, c->nb_bnd, c->partial_bgt.p,
                                         c->nb_bnd, c->partial_vp.p, c->nb_vp, c->scalars.p);
  check_launch(c);
}

// 2D FFT of the P x P array z (rows, transpose into t, rows): the spectrum
// ends in t in transposed layout [k_col][k_row].  The inverse takes t in that
// layout and leaves the result in z in the original layout.
// 2D FFT of a P x P array: rows of `first`, transpose into `second`, rows of
// `second` (so the spectrum is transposed; the inverse undoes it).  Only the
// first rows_in rows of `first` can be non-zero (the transform of a zero row is
// zero, so the others are left as they are), and only the first rows_out rows
// of the result are needed (the transpose and the last pass stop there).
void fft2(sc_ctx *c, double2 *z, double2 *t, int inverse, int rows_in, int rows_out) {
  const int P = c->fft_p;
  const int thr = std::min(P / 2, 512);
  const size_t smem = 2 * (size_t)P * sizeof(double2);
  const dim3 tb(32, 8), tg((rows_out + 31) / 32, P / 32);
  double2 *first = inverse ? t : z, *second = inverse ? z : t;
  k_fft_rows<<<rows_in, thr, smem, c->stream>>>(c->fft_plan, P, (const double2 *)c->fft_tw.p, first, inverse);
  check_launch(c);
  k_fft_transpose<<<tg, tb, 0, c->stream>>>(P, first, second);
  check_launch(c);
  k_fft_rows<<<rows_out, thr, smem, c->stream>>>(c->fft_plan, P, (const double2 *)c->fft_tw.p, second, inverse);
  check_launch(c);
}

void poisson(sc_ctx *c, const double *j, double *a_out, int mean_from_scalars) {
  const HostSetup &S = c->S;
  const int n = S.n0;
  const size_t nn2 = 2 * c->nn0();
  if (mean_from_scalars) {
    k_subtract_mean<<<grid1(nn2, 256), 256, 0, c->stream>>>(
        n, j, (const double *)c->scalars.p, (int)(offsetof(Scalars, j_mean) / sizeof(double)),
        c->pois_s.p);
    check_launch(c);
  } else {
    CUDA_TRY(cudaMemcpyAsync(c->pois_s.p, j, nn2 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
  }
  ProfScope prof(c, 2);
  const int P = c->fft_p;
  const size_t pp = (size_t)P * P;
  double2 *z = (double2 *)c->fft_z.p, *t = (double2 *)c->fft_t.p;
  k_fft_pack<<<grid1(pp, 256), 256, 0, c->stream>>>(n, P, c->pois_s.p, z);
  check_launch(c);
  fft2(c, z, t, 0, n, P);  // the current fills rows < N0 of z
  k_fft_mul<<<grid1(pp, 256), 256, 0, c->stream>>>(pp, (const double2 *)c->fft_kf.p, t);
  check_launch(c);
  fft2(c, z, t, 1, P, n);  // A is read from rows < N0 of z
  k_fft_unpack<<<grid1(c->nn0(), 256), 256, 0, c->stream>>>(n, P, 1.0 / ((double)P * (double)P), z, a_out);
  check_launch(c);
}

// The kernel K(u, v) = -h^2 scale sum_k (+/-) f_k(u) f_k(v), reflected
// (A is a correlation, the FFT product a convolution) and wrapped into the
// P x P array, and its spectrum in the transposed layout of fft2.
void poisson_setup(sc_ctx *c) {
  const HostSetup &S = c->S;
  const int n = S.n0;
  // The smallest side P >= 2 N0 - 1 of the form 32 * 2^a 3^b 5^c (a multiple
  // of the 32-wide transpose tiles whose rows the mixed-radix FFT handles).
  auto smooth = [](int m) {
    for (int f : {2, 3, 5})
      while (m % f == 0) m /= f;
    return m == 1;
  };
  int m = 1;
  while (32 * m < 2 * n - 1 || !smooth(m)) ++m;
  const int P = 32 * m;
  if (P > 4096) throw EngineError(SC_ERR_ARG, "lattice too large for the Poisson transform (N0 > 2048)");
  c->fft_p = P;
  FftPlan plan{};
  {
    int r = P, twos = 0;
    while (r % 2 == 0) r /= 2, ++twos;
    for (int k = 0; k < twos / 2; ++k) plan.radix[plan.n_stages++] = 4;
    if (twos % 2) plan.radix[plan.n_stages++] = 2;
    while (r % 3 == 0) r /= 3, plan.radix[plan.n_stages++] = 3;
    while (r % 5 == 0) r /= 5, plan.radix[plan.n_stages++] = 5;
  }
  c->fft_plan = plan;
  std::vector<double> tw(2 * (size_t)P);  // exp(-2 pi i q / P), q < P
  for (int q = 0; q < P; ++q) {
    const double ang = -2.0 * M_PI * (double)q / (double)P;
    tw[2 * q] = std::cos(ang);
    tw[2 * q + 1] = std::sin(ang);
  }
  c->fft_tw.upload(tw, c->stream);
  const size_t pp = (size_t)P * P;
  std::vector<double> kr(2 * pp, 0.0);
  const double factor = -1.0 * (S.h * S.h) * S.vp_scale;
  const int nf = 2 * n - 1;
  for (int k = 0; k < S.n_filters; ++k) {
    const double *f = &S.filters[(size_t)k * nf];  // f_k(u) = f[u + n - 1]
    const double sgn = S.filter_pos[k] ? factor : -factor;
    for (int u = -(n - 1); u <= n - 1; ++u) {
      const double fu = sgn * f[u + n - 1];
      const size_t row = (size_t)((-u + P) % P) * P;
      for (int v = -(n - 1); v <= n - 1; ++v) kr[2 * (row + (size_t)((-v + P) % P))] += fu * f[v + n - 1];
    }
  }
  c->fft_z.alloc(2 * pp);
  c->fft_t.alloc(2 * pp);
  c->fft_kf.alloc(2 * pp);
  CUDA_TRY(cudaMemcpyAsync(c->fft_z.p, kr.data(), 2 * pp * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  if (2 * P * sizeof(double2) > 48 * 1024)
    CUDA_TRY(cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * P * sizeof(double2))));
  fft2(c, (double2 *)c->fft_z.p, (double2 *)c->fft_kf.p, 0, P, P);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
}

void accelerate(sc_ctx *c) {
  const HostSetup &S = c->S;
  AccConsts C{};
  C.kind = S.acc.kind;
  C.nf = c->n_fields();
  C.step_size = S.acc.step_size;
  C.factor = S.acc.step_size_factor;
  C.mincos = S.acc.cos_similarity_min;
  C.smax = S.acc.step_size_max;
  C.smin = S.acc.step_size_min;
  C.drag = S.acc.drag;
  const size_t nn = c->nn0();
  if (C.kind == ACC_ANDERSON) {
    const size_t tot = (size_t)C.nf * nn;
    const int rank = S.acc.rank;
    k_and_store<<<c->nb_acc, REDUCE_THREADS, 0, c->stream>>>(tot, rank, c->xstate.p, c->gstate.p, c->and_x.p,
                                                             c->and_d.p, c->acc_state.p, c->partial_acc.p);
    check_launch(c);
    k_and_solve<<<1, 256, 0, c->stream>>>(rank, c->partial_acc.p, c->nb_acc, c->acc_state.p);
    check_launch(c);
    k_and_update<<<grid1(tot, 256), 256, 0, c->stream>>>(tot, rank, C.step_size, c->and_x.p, c->and_d.p,
                                                         c->acc_state.p, c->xstate.p);
    check_launch(c);
    return;
  }
  if (C.kind == ACC_CONGACC || C.kind == ACC_BB) {
    dim3 grid(c->nb_acc, C.nf);
    k_acc_sums<<<grid, REDUCE_THREADS, 0, c->stream>>>(C.nf, nn, c->xstate.p, c->gstate.p, c->acc_m.p,
                                                        c->partial_acc.p);
    check_launch(c);
    k_acc_scalars<<<1, 256, 0, c->stream>>>(C, c->partial_acc.p, c->nb_acc, c->acc_state.p);
    check_launch(c);
  }
  k_acc_update<<<grid1((size_t)C.nf * nn, 256), 256, 0, c->stream>>>(C, nn, c->gstate.p, c->xstate.p,
                                                                       c->acc_m.p, c->acc_state.p);
  check_launch(c);
}

// Frame extension and rotation back of one swept chunk.
int chunk_pair(const sc_ctx *c, const Chunk &ch) {
  return (c->pair && ch.a_begin == 0 && ch.a_end == c->S.n_angles) ? c->pair : 0;
}
// Frame slots of a chunk: with mirrored pairs only the first half is stored.
int chunk_slots(const sc_ctx *c, const Chunk &ch) {
  return chunk_pair(c, ch) ? c->pair : ch.a_end - ch.a_begin;
}

template <typename R>
void frame_to_reference(sc_ctx *c, const Chunk &ch) {
  using Fr = typename FrameOf<R>::type;
  const HostSetup &S = c->S;
  const int pair = chunk_pair(c, ch);
  const int a_stored = ch.a_begin + chunk_slots(c, ch);
  const int h0 = S.halo_angle_off[ch.a_begin], h1 = S.halo_angle_off[a_stored];
  if (h1 > h0) {
    k_halo<<<grid1(h1 - h0, 128), 128, 0, c->stream>>>(h1 - h0, h0, S.n1, c->halo_angle.p, ch.a_begin,
                                                        c->halo_site.p, c->halo_off.p, c->halo_src.p,
                                                        (Fr *)c->w_fr);
    check_launch(c);
  }
  // A warp covers an 8 x 4 patch of the reference grid (its rotated corners
  // share cache lines of the frame).
  dim3 blk(8, 32), grid((S.n0 + 7) / 8, (S.n0 + 31) / 32);
  ProfScope prof(c, 1);
  auto kern = S.nc == 1 ? k_rotate_back<Fr, 1> : S.nc == 2 ? k_rotate_back<Fr, 2> : k_rotate_back<Fr, 0>;
  kern<<<grid, blk, 0, c->stream>>>(S.n0, S.n1, S.nc, ch.a_begin, a_stored, pair, c->ang.p, (const Fr *)c->w_fr,
                                    c->acc_d.p, c->acc_j.p, c->acc_fe.p);
  check_launch(c);
}

// Lanes per reference site: the smallest of 8, 16, 32 that holds the block's
// energies (more energies take several blocks along z).
template <typename LF>
static void launch_rotate_back_ldos(sc_ctx *c, const Chunk &ch) {
  const HostSetup &S = c->S;
  auto go = [&](auto kern, int el, int tx) {
    const int ty = 256 / el / tx;
    dim3 grid((S.n0 + tx - 1) / tx, (S.n0 + ty - 1) / ty, (S.ne + el - 1) / el);
    kern<<<grid, 256, 0, c->stream>>>(S.n0, S.n1, S.ne, ch.a_begin, ch.a_end, c->ang.p, (const LF *)c->ldf.p,
                                      c->ldos_acc.p);
  };
  if (S.ne <= 8)
    go(k_rotate_back_ldos<8, 8, LF>, 8, 8);
  else if (S.ne <= 16)
    go(k_rotate_back_ldos<16, 4, LF>, 16, 4);
  else
    go(k_rotate_back_ldos<32, 4, LF>, 32, 4);
  check_launch(c);
}

template <typename R>
void run_chunks_ldos(sc_ctx *c, int burn_in) {
  const HostSetup &S = c->S;
  // The LDOS frame buffer is not cleared between chunks or iterations: the
  // sweep rewrites every grain site of the chunk's angles and the extension
  // every site next to the grain, and those are the only frame sites that the
  // bilinear rotation back reads for a site inside the grain; sites outside
  // the grain may read values left by other angles, and k_ldos_finalize
  // discards them.  (The buffer is zeroed once at creation, so every value in
  // it is finite.)  Clearing 32 energies x N1^2 sites for every angle cost
  // about as much as the sweep itself on large grains.
  for (const Chunk &ch : c->chunks) {
    launch_sweep<R>(c, ch, burn_in);
    if (burn_in) continue;
    const int h0 = S.halo_angle_off[ch.a_begin], h1 = S.halo_angle_off[ch.a_end];
    if (h1 > h0) {
      using LF = typename LdosOf<R>::type;
      k_halo_ldos<LF><<<grid1((size_t)(h1 - h0) * S.ne, 128), 128, 0, c->stream>>>(
          h1 - h0, h0, S.n1, S.ne, c->halo_angle.p, ch.a_begin, c->halo_site.p, c->halo_off.p, c->halo_src.p,
          (LF *)c->ldf.p);
      check_launch(c);
    }
    ProfScope prof(c, 1);
    launch_rotate_back_ldos<typename LdosOf<R>::type>(c, ch);
  }
}

template <typename R>
void run_chunks(sc_ctx *c, int burn_in) {
  const HostSetup &S = c->S;
  const size_t nn1 = (size_t)S.n1 * S.n1;
  if (S.keldysh) {
    run_chunks_ldos<R>(c, burn_in);
    return;
  }
  const bool clear = c->chunks.size() > 1 || !c->frames_zeroed;
  for (const Chunk &ch : c->chunks) {
    const int nslots = chunk_slots(c, ch);
    if (!burn_in && clear) {
      CUDA_TRY(cudaMemsetAsync(c->w_fr, 0, (size_t)nslots * nn1 * c->frame_rec(), c->stream));
      c->frames_zeroed = c->chunks.size() == 1;
    }
    launch_sweep<R>(c, ch, burn_in);
    if (burn_in) continue;
    frame_to_reference<R>(c, ch);
  }
}

// Context::compute in three parts: before the sweep (accelerator step,
// extended order parameter, cleared accumulators), the sweep with the frame
// rotation, and after it (finalize, boundary condition, vector potential).
template <typename R>
void compute_pre(sc_ctx *c) {
  if (!c->first_compute) accelerate(c);
  if (!c->boundary_initialized) boundary_initial<R>(c);
  extend_reference(c);
  c->acc_d.zero(c->stream);
  c->acc_j.zero(c->stream);
  c->acc_fe.zero(c->stream);
}

template <typename R>
void compute_post(sc_ctx *c);

template <typename R>
void compute_once(sc_ctx *c) {
  compute_pre<R>(c);
  run_chunks<R>(c, 0);
  compute_post<R>(c);
}

// One Context::compute iteration; once the iteration is steady (after the
// first one, boundary values set, frames cleared) it is captured as a CUDA
// graph and replayed, so a small grain pays one graph launch instead of ~25
// kernel launches per iteration.
template <typename R>
void compute_iteration(sc_ctx *c) {
  static const bool no_graph = std::getenv("SCB_NO_GRAPH") != nullptr;
  const bool steady = !c->first_compute && c->boundary_initialized && (c->frames_zeroed || c->chunks.size() > 1) &&
                      !c->profiling && !c->batch_member && !c->iter_graph_failed && !no_graph;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(c->stream, &cap));
  if (cap != cudaStreamCaptureStatusNone) {  // a caller's capture records the launches (sc_compute checked
    compute_once<R>(c);                      // that the iteration is steady); the own graph stays valid
    return;
  }
  if (!steady) {
    c->drop_graph();
    compute_once<R>(c);
    return;
  }
  if (!c->iter_graph) {
    const long long l0 = c->launches;
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      compute_once<R>(c);
    } catch (...) {
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CUDA_TRY(cudaStreamEndCapture(c->stream, &g));
    const cudaError_t e = cudaGraphInstantiate(&c->iter_graph, g, 0);
    cudaGraphDestroy(g);
    c->iter_graph_launches = c->launches - l0;
    c->launches = l0;
    if (e != cudaSuccess) {  // run eagerly from now on (nothing of the capture ran)
      (void)cudaGetLastError();
      c->iter_graph = nullptr;
      c->iter_graph_failed = true;
      compute_once<R>(c);
      return;
    }
  }
  CUDA_TRY(cudaGraphLaunch(c->iter_graph, c->stream));
  c->launches += c->iter_graph_launches;
}

template <typename R>
void compute_post(sc_ctx *c) {
  const HostSetup &S = c->S;
  const size_t nn = c->nn0();
  // Finalize.
  {
    double *delta = c->xstate.p, *avec = c->xstate.p + (size_t)2 * S.nc * nn;
    double *delta_new = c->gstate.p;
    const double jfactor = (double)(2 * S.charge_sign) * S.temperature;
    k_finalize<<<c->nb_fin, REDUCE_THREADS, 0, c->stream>>>(
        S.n0, S.nc, S.h, jfactor, c->has_vp() ? 1 : 0, c->dom.p, c->coupling.p, c->acc_d.p, c->acc_j.p,
        c->acc_fe.p, delta, avec, delta_new, c->j_real.p, c->partial_fin.p);
    check_launch(c);
    FinalizeConsts F{};
    F.nc = S.nc;
    F.norm = S.norm;
    F.n_grain = S.n_grain;
    F.has_vp = c->has_vp() ? 1 : 0;
    F.n_elem_field = 2 * nn;
    F.temperature = S.temperature;
    F.h = S.h;
    F.lambda = S.lambda;
    F.conv = S.conv_crit;
    double si = 0.0;
    for (int e = 0; e < S.ne; ++e) si += S.residues[e] / S.e_im[e];
    F.sum_inv = si * S.temperature;
    for (int k = 0; k < S.nc; ++k) F.log_t_tc[k] = std::log(S.temperature / S.tc[k]);
    k_scalars_a<<<1, 256, 0, c->stream>>>(F, c->partial_fin.p, c->nb_fin, c->scalars.p);
    check_launch(c);
  }
  boundary_condition<R>(c);
  if (c->has_vp()) {
    double *a_new = c->gstate.p + (size_t)2 * S.nc * nn;
    const double *avec = c->xstate.p + (size_t)2 * S.nc * nn;
    poisson(c, c->j_real.p, a_new, 1);
    k_residual<<<c->nb_vp, REDUCE_THREADS, 0, c->stream>>>(2 * nn, avec, a_new, c->partial_vp.p);
    check_launch(c);
  }
  launch_scalars_b(c, 1, c->has_vp() ? 1 : 0, 1);
  c->first_compute = false;
}

void ldos_begin_block(sc_ctx *c, int b);

template <typename R>
void burn_in_once(sc_ctx *c) {
  if (c->S.keldysh && c->ldos_block < 0) ldos_begin_block(c, 0);
  if (!c->boundary_initialized) boundary_initial<R>(c);
  extend_reference(c);
  run_chunks<R>(c, 1);
  boundary_condition<R>(c);
  launch_scalars_b(c, 1, 0, 0);
}

// Energies of LDOS block b and fresh homogeneous boundary values
// (IntegrationIteratorKeldysh.h:250-268: a new energy interval re-initialises
// the Riccati solver and the boundary).
void ldos_begin_block(sc_ctx *c, int b) {
  const HostSetup &S = c->S;
  if (b < 0 || b >= S.ldos_n_blocks) throw EngineError(SC_ERR_ARG, "LDOS block out of range");
  std::vector<double> e;
  ldos_block_energies(S, b, e);
  CUDA_TRY(cudaMemcpyAsync(c->e_re.p, e.data(), e.size() * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  c->ldos_block = b;
  c->boundary_initialized = false;
}

int ldos_block_count(const sc_ctx *c, int b) {
  const int n = (int)c->S.ldos_energies.size();
  return std::min(c->S.ldos_block, n - b * c->S.ldos_block);
}

// One LDOS iteration of the current block (IntegrationIteratorKeldysh::compute
// with inIsBurnIn = false, IntegrationIteratorKeldysh.h:300-389).
template <typename R>
void ldos_once(sc_ctx *c) {
  const HostSetup &S = c->S;
  if (c->ldos_block < 0) ldos_begin_block(c, 0);
  if (!c->boundary_initialized) boundary_initial<R>(c);
  extend_reference(c);
  c->ldos_acc.zero(c->stream);
  run_chunks<R>(c, 0);
  boundary_condition<R>(c);
  const int nf = ldos_block_count(c, c->ldos_block);
  double *blk = c->ldos_all.p + (size_t)c->ldos_block * S.ldos_block * c->nn0();
  k_ldos_finalize<<<c->nb_vp, 256, 0, c->stream>>>(S.n0, nf, c->dom.p, c->ldos_acc.p, blk, c->partial_vp.p);
  check_launch(c);
  launch_scalars_b(c, 1, 1, 0, (size_t)nf * c->nn0());
}

// Whether the caller is capturing the context's stream into a CUDA graph.
bool stream_captured(sc_ctx *c) {
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CUDA_TRY(cudaStreamIsCapturing(c->stream, &cap));
  return cap != cudaStreamCaptureStatusNone;
}

void read_scalars(sc_ctx *c) {
  CUDA_TRY(cudaMemcpyAsync(&c->host_scalars, c->scalars.p, sizeof(Scalars), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
}

// Chunking of the angles so that the sweep scratch and the frame buffers stay
// within a device-memory budget.
void plan_chunks(sc_ctx *c, std::vector<int4> &items) {
  const HostSetup &S = c->S;
  const int n1 = S.n1, na = S.n_angles;
  std::vector<int> kmax(na, 0), count(na, 0);
  std::vector<std::vector<int4>> per(na);
  for (int a = 0; a < na; ++a)
    for (int x = S.x0[a]; x <= S.x1[a]; ++x) {
      const int lo = S.col_lo[(size_t)a * n1 + x], hi = S.col_hi[(size_t)a * n1 + x];
      if (lo < 0) continue;
      per[a].push_back(make_int4(a, x, lo, hi));
      kmax[a] = std::max(kmax[a], hi - lo + 1);
    }
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  double budget_mb = 0.35 * (double)free_b / 1048576.0;
  if (const char *env = std::getenv("SCB_SCRATCH_MB")) budget_mb = std::atof(env);
  // A batch grain sweeps all its angles in one chunk (the batch pools memory).
  const double budget = c->batch_member ? 1e300 : budget_mb * 1048576.0;
  const size_t per_row = (size_t)c->e_pass * c->esize() + 3 * sizeof(double);
  const size_t frame_slot = S.keldysh ? (size_t)n1 * n1 * S.ne * c->ldos_esize()
                                      : (size_t)n1 * n1 * 2 * sizeof(double2);
  items.clear();
  if (c->pair) {
    // One chunk over all angles; only the first half gets trajectory columns.
    Chunk ch{0, na, 0, 0, 0};
    for (int b = 0; b < na / 2; ++b) {
      items.insert(items.end(), per[b].begin(), per[b].end());
      ch.kmax = std::max(ch.kmax, kmax[b]);
    }
    ch.item_end = (int)items.size();
    const double need = (double)items.size() * ch.kmax * per_row + (double)(na / 2) * frame_slot;
    if (need <= budget) {
      c->chunks.push_back(ch);
      return;
    }
    c->pair = 0;  // does not fit one chunk: sweep every angle
    items.clear();
  }
  int a = 0;
  while (a < na) {
    Chunk ch{a, a, (int)items.size(), (int)items.size(), 0};
    size_t nitems = 0;
    while (a < na) {
      const int k2 = std::max(ch.kmax, kmax[a]);
      const size_t n2 = nitems + per[a].size();
      const double need = (double)n2 * k2 * per_row + (double)(a - ch.a_begin + 1) * frame_slot;
      if (a > ch.a_begin && need > budget) break;
      ch.kmax = k2;
      nitems = n2;
      items.insert(items.end(), per[a].begin(), per[a].end());
      ++a;
    }
    ch.a_end = a;
    ch.item_end = (int)items.size();
    c->chunks.push_back(ch);
  }
}

void upload_static(sc_ctx *c) {
  HostSetup &S = c->S;
  cudaStream_t s = c->stream;
  const int na = S.n_angles;
  std::vector<AngleParams> ap(na);
  for (int a = 0; a < na; ++a) {
    AngleParams &p = ap[a];
    p.cD = S.cD[a];
    p.sD = S.sD[a];
    p.cA = S.cA[a];
    p.sA = S.sA[a];
    p.cB = S.cB[a];
    p.sB = S.sB[a];
    p.cE = S.cE[a];
    p.sE = S.sE[a];
    p.vx = S.vx[a];
    p.vy = S.vy[a];
    p.w = S.weight[a];
    p.hs = S.step[a];
    p.sx = S.vx[a] * S.weight[a];
    p.sy = S.vy[a] * S.weight[a];
    for (int k = 0; k < MAX_COMP; ++k) p.eta[k] = k < S.nc ? S.eta[(size_t)a * S.nc + k] : 0.0;
  }
  c->ang.upload(ap, s);
  c->labels.upload(S.labels, s);
  c->dom.upload(S.domain_ref, s);
  c->idx_in_g.upload(S.idx_in_g, s);
  c->idx_out_g.upload(S.idx_out_g, s);
  c->idx_in_gt.upload(S.idx_in_gt, s);
  c->idx_out_gt.upload(S.idx_out_gt, s);
  c->dist_in_g.upload(S.dist_in_g, s);
  c->dist_out_g.upload(S.dist_out_g, s);
  c->dist_in_gt.upload(S.dist_in_gt, s);
  c->dist_out_gt.upload(S.dist_out_gt, s);
  c->bc_src_g.upload(S.bc_g.src, s);
  c->bc_w_g.upload(S.bc_g.w, s);
  c->bc_ws_g.upload(S.bc_g.wsum, s);
  c->bc_src_gt.upload(S.bc_gt.src, s);
  c->bc_w_gt.upload(S.bc_gt.w, s);
  c->bc_ws_gt.upload(S.bc_gt.wsum, s);
  c->halo_site.upload(S.halo_site, s);
  c->halo_off.upload(S.halo_src_off, s);
  c->halo_src.upload(S.halo_src, s);
  std::vector<int> hang(S.halo_site.size());
  for (int a = 0; a < na; ++a)
    for (int k = S.halo_angle_off[a]; k < S.halo_angle_off[a + 1]; ++k) hang[k] = a;
  c->halo_angle.upload(hang, s);
  c->rext_site.upload(S.rext_site, s);
  c->rext_off.upload(S.rext_src_off, s);
  c->rext_src.upload(S.rext_src, s);
  c->e_re.upload(S.e_re, s);
  c->e_im.upload(S.e_im, s);
  c->res.upload(S.residues, s);
  c->coupling.upload(S.coupling, s);
  if (S.n_filters) {
    c->filters.upload(S.filters, s);
    c->filter_pos.upload(S.filter_pos, s);
  }
  // Exit nodes (for the homogeneous initial boundary values).
  std::vector<int> ag, xg, yg, agt, xgt, ygt;
  ag.resize(S.n_out_g);
  xg.resize(S.n_out_g);
  yg.resize(S.n_out_g);
  agt.resize(S.n_out_gt);
  xgt.resize(S.n_out_gt);
  ygt.resize(S.n_out_gt);
  const int n1 = S.n1;
  for (int a = 0; a < na; ++a)
    for (int x = 0; x < n1; ++x) {
      const size_t ax = (size_t)a * n1 + x;
      if (S.idx_out_g[ax] >= 0)
        for (int k = 0; k < S.nisect_g[ax]; ++k) {
          const int o = S.idx_out_g[ax] + k;
          ag[o] = a;
          xg[o] = x;
          yg[o] = S.coord_g[o];
        }
      if (S.idx_out_gt[ax] >= 0)
        for (int k = 0; k < S.nisect_gt[ax]; ++k) {
          const int o = S.idx_out_gt[ax] + k;
          agt[o] = a;
          xgt[o] = x;
          ygt[o] = S.coord_gt[o];
        }
    }
  c->onode_a_g.upload(ag, s);
  c->onode_x_g.upload(xg, s);
  c->onode_y_g.upload(yg, s);
  c->onode_a_gt.upload(agt, s);
  c->onode_x_gt.upload(xgt, s);
  c->onode_y_gt.upload(ygt, s);

  // Mirror pairing of angle a with a + n/2 (mixed mode only, circular Fermi
  // surface): every frame of the second half must be the 180-degree mirror of
  // its partner, with entry and exit labels exchanged.  All four basis
  // symmetries are even, so the order parameter is the same on both angles.
  c->pair = 0;
  if (c->mode == SC_MODE_MIXED && !S.keldysh && !S.fs_tight_binding && na % 2 == 0 &&
      !std::getenv("SCB_NO_PAIRING")) {
    const int n1p = S.n1;
    const size_t nn1p = (size_t)n1p * n1p;
    bool ok = true;
    for (int a = 0; a < na / 2 && ok; ++a) {
      const uint8_t *la = &S.labels[(size_t)a * nn1p];
      const uint8_t *lb = &S.labels[(size_t)(a + na / 2) * nn1p];
      for (int y = 0; y < n1p && ok; ++y)
        for (int x = 0; x < n1p; ++x) {
          uint8_t v = la[(size_t)y * n1p + x];
          if (v == 2) v = 3;
          else if (v == 3) v = 2;
          if (lb[(size_t)(n1p - 1 - y) * n1p + (n1p - 1 - x)] != v) {
            ok = false;
            break;
          }
        }
    }
    if (ok) c->pair = na / 2;
  }
  c->e_pass = S.ne <= SWEEP_MAX_ENERGIES ? S.ne : ENERGY_PASS;
  std::vector<int4> items;
  plan_chunks(c, items);
  c->items.upload(items, s);
  c->h_items = items;  // host copy: the batch plans its work units from it
  // Energy groups per column.
  c->groups = 1;
  c->log_groups = 0;
  const char *eg = std::getenv("SCB_ENERGY_GROUPS");
  // Default (fastest measured on B200 for 7-14 Ozaki energies): the fewest
  // threads per column that keep at most four energies per thread; three
  // (FP64) or four (mixed) resident blocks per SM.  Mixed precision prefers an
  // even count, which the packed FP32 sweep takes in pairs (C2, 14 energies:
  // four threads of four energies, sweep 5.70 ms, against eight threads of two
  // 6.07 ms).
  const bool fp32_sweep = c->mode == SC_MODE_MIXED && !S.keldysh;
  const int per_thread = 4;
  int want = 1;
  if (eg) want = std::atoi(eg);
  else {
    while ((c->e_pass + want - 1) / want > per_thread && want < 8) want *= 2;
    // Small grains: too few trajectory columns to fill the GPU twice over,
    // so spread the energies over more threads per column.
    int dev = 0, n_sm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
    const double resident = (double)n_sm * (fp32_sweep ? 4 : 3) * 128;
    size_t max_items = 0;
    for (const Chunk &ch : c->chunks) max_items = std::max(max_items, (size_t)(ch.item_end - ch.item_begin));
    while ((double)max_items * want < 2.0 * resident && want < 8 && (c->e_pass + want - 1) / want > 1) want *= 2;
    const int ept_w = (c->e_pass + want - 1) / want;
    if (fp32_sweep && ept_w > 1 && ept_w % 2 == 1 && want < 8) want *= 2;
  }
  while (c->groups < want && c->groups < 8) {
    c->groups *= 2;
    c->log_groups++;
  }
  c->ept = (c->e_pass + c->groups - 1) / c->groups;
  if (c->ept > 16) throw EngineError(SC_ERR_ARG, "too many Ozaki energies per thread");
  c->emax2 = fp32_sweep ? !std::getenv("SCB_SWEEP_EMAX4") : std::getenv("SCB_SWEEP_EMAX2") != nullptr;

  // State and work buffers.
  const size_t nn = c->nn0();
  const int nf = c->n_fields();
  c->xstate.alloc((size_t)(2 * S.nc + 2) * nn);
  c->gstate.alloc((size_t)(2 * S.nc + 2) * nn);
  c->xstate.zero(s);
  c->gstate.zero(s);
  c->rfields.alloc((size_t)2 * (S.nc + 1) * nn);
  if (c->mode == SC_MODE_MIXED) c->rfields32.alloc((size_t)(S.nc + 1) * nn + 1);
  c->j_real.alloc(2 * nn);
  c->j_real.zero(s);
  c->acc_d.alloc((size_t)2 * S.nc * nn);
  c->acc_j.alloc(2 * nn);
  c->acc_fe.alloc(nn);
  size_t off = 0;
  for (int w = 0; w < 4; ++w) {
    c->bnd_off[w] = off;
    off += (size_t)c->n_bnd(w) * S.ne * c->esize();
    off = (off + 255) & ~size_t(255);
  }
  c->bnd.alloc(off / sizeof(double) + 1);
  c->bnd.zero(s);
  size_t scr = 0, scr2 = 0;
  int max_slots = 1;
  for (const Chunk &ch : c->chunks) {
    const size_t ni = (size_t)(ch.item_end - ch.item_begin);
    const size_t ni32 = (ni + 31) / 32 * 32;  // whole scratch tiles
    // Energies per row rounded up to even: the packed FP32 sweep stores them in pairs.
    scr = std::max(scr, ni32 * ch.kmax * (size_t)((c->e_pass + 1) & ~1) * c->esize());
    scr2 = std::max(scr2, ni32 * ch.kmax * 4);
    max_slots = std::max(max_slots, chunk_slots(c, ch));
  }
  c->need_scratch = scr + 8;
  c->need_scratch2 = (scr2 + 1) * sizeof(double);
  c->need_frame = (size_t)max_slots * n1 * n1 * c->frame_rec();
  if (c->batch_member) {
    // Work buffers come from the batch's pool.
  } else if (S.keldysh) {
    c->scratch.alloc(scr / sizeof(double) + 1);
    c->scratch2.alloc(scr2 + 1);
    c->w_scratch = c->scratch.p;
    c->w_scratch2 = c->scratch2.p;
    c->ldf.alloc(((size_t)max_slots * S.ne * n1 * n1 * c->ldos_esize() + 7) / 8);  // as doubles
    c->ldf.zero(s);  // once: afterwards every slot holds finite values (see run_chunks_ldos)
    c->ldos_acc.alloc((size_t)S.ne * nn);
    c->ldos_all.alloc((size_t)S.ldos_n_blocks * S.ldos_block * nn);
    c->ldos_all.zero(s);
  } else {
    c->scratch.alloc(scr / sizeof(double) + 1);
    c->scratch2.alloc(scr2 + 1);
    c->w_scratch = c->scratch.p;
    c->w_scratch2 = c->scratch2.p;
    c->frames.alloc((size_t)max_slots * n1 * n1 * 4);  // FP64-sized records (the adjoint's buffers too)
    c->w_fr = c->frames.p;
  }
  c->nb_fin = std::min<int>(592, (int)grid1(nn, REDUCE_THREADS));
  c->nb_bnd = std::min<int>(592, (int)grid1((size_t)std::max(S.n_in_g, S.n_in_gt) * S.ne, REDUCE_THREADS));
  c->nb_vp = std::min<int>(296, (int)grid1(2 * nn, REDUCE_THREADS));
  c->nb_acc = std::min<int>(148, (int)grid1(nn, REDUCE_THREADS));
  c->partial_fin.alloc((size_t)c->nb_fin * NQ);
  c->partial_bg.alloc((size_t)c->nb_bnd * 6);
  c->partial_bgt.alloc((size_t)c->nb_bnd * 6);
  c->partial_vp.alloc((size_t)c->nb_vp * 6);
  c->partial_acc.alloc((size_t)16 * c->nb_acc * 3);
  c->partial_vp.zero(s);
  if (S.n_filters && !S.keldysh) {
    c->pois_s.alloc(2 * nn);
    poisson_setup(c);
  }
  c->acc_m.alloc((size_t)std::max(nf, 1) * nn);
  c->acc_m.zero(s);
  if (S.acc.kind == ACC_ANDERSON) {
    if (S.acc.rank < 1 || S.acc.rank > AND_MAX_RANK) throw EngineError(SC_ERR_ARG, "Anderson rank must be 1..16");
    c->and_x.alloc((size_t)S.acc.rank * nf * nn);
    c->and_d.alloc((size_t)S.acc.rank * nf * nn);
  }
  c->acc_state.alloc(1);
  c->acc_state.zero(s);
  c->scalars.alloc(1);
  Scalars init{};
  init.first_j = 1;
  init.first_fe = 1;
  CUDA_TRY(cudaMemcpyAsync(c->scalars.p, &init, sizeof(Scalars), cudaMemcpyHostToDevice, s));
  c->tmp_io.alloc((size_t)(2 * S.nc + 2) * nn);
  CUDA_TRY(cudaStreamSynchronize(s));
}

int fail(sc_ctx *c, const EngineError &e) {
  if (c) c->err = e.msg;
  else g_create_error = e.msg;
  return e.code;
}

#define API_BEGIN try {
#define API_END                                              \
  }                                                          \
  catch (const EngineError &e) { return fail(ctx, e); }      \
  catch (const std::exception &e) {                          \
    return fail(ctx, EngineError(SC_ERR_ARG, e.what()));     \
  }                                                          \
  return SC_OK;

}  // namespace

extern "C" {

}  // extern "C"

namespace {
// Shared part of sc_create / sc_ldos_create: the setup is built by `make`.
template <typename F>
int create_context(int mode, sc_ctx **out, F make) {
  if (!out) {
    g_create_error = "null output handle";
    return SC_ERR_ARG;
  }
  *out = nullptr;
  if (mode != SC_MODE_FP64 && mode != SC_MODE_MIXED) {
    g_create_error = "mode must be SC_MODE_FP64 or SC_MODE_MIXED";
    return SC_ERR_ARG;
  }
  sc_ctx *c = new sc_ctx();
  c->mode = mode;
  try {
    const std::string e = make(c->S);
    if (!e.empty()) throw EngineError(SC_ERR_ARG, e);
    if (c->S.nc > MAX_COMP) throw EngineError(SC_ERR_ARG, "at most 4 order-parameter components");
    if (2 * c->S.nc + 2 > 16) throw EngineError(SC_ERR_ARG, "too many accelerator fields");
    CUDA_TRY(cudaGetDevice(&c->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    upload_static(c);
  } catch (const EngineError &e) {
    g_create_error = e.msg;
    cudaStream_t s = c->own_stream;
    delete c;
    if (s) cudaStreamDestroy(s);
    return e.code;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    cudaStream_t s = c->own_stream;
    delete c;
    if (s) cudaStreamDestroy(s);
    return SC_ERR_ARG;
  }
  *out = c;
  return SC_OK;
}
}  // namespace

extern "C" {

int sc_create(const char *config_json, int mode, sc_ctx **out) {
  if (!config_json) {
    g_create_error = "sc_create: null argument";
    return SC_ERR_ARG;
  }
  return create_context(mode, out, [&](HostSetup &S) { return build_setup(config_json, S); });
}

int sc_ldos_create(const char *simulation_json, const char *postprocess_json, int mode, sc_ctx **out) {
  if (!simulation_json || !postprocess_json) {
    g_create_error = "sc_ldos_create: null argument";
    return SC_ERR_ARG;
  }
  return create_context(mode, out, [&](HostSetup &S) {
    return build_ldos_setup(simulation_json, postprocess_json, S);
  });
}

int sc_destroy(sc_ctx *ctx) {
  if (!ctx) return SC_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  cudaStream_t s = ctx->own_stream;
  delete ctx;  // device arrays free themselves
  if (s) cudaStreamDestroy(s);
  return SC_OK;
}

const char *sc_last_error(const sc_ctx *ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int sc_get_dims(const sc_ctx *ctx, int *n0, int *n1, int *n_angles, int *n_energies, int *n_comp) {
  if (!ctx) return SC_ERR_ARG;
  if (n0) *n0 = ctx->S.n0;
  if (n1) *n1 = ctx->S.n1;
  if (n_angles) *n_angles = ctx->S.n_angles;
  if (n_energies) *n_energies = ctx->S.ne;
  if (n_comp) *n_comp = ctx->S.nc;
  return SC_OK;
}

int sc_site_updates(const sc_ctx *ctx, long long *per_iteration) {
  if (!ctx || !per_iteration) return SC_ERR_ARG;
  *per_iteration = ctx->S.site_updates_per_iteration();
  return SC_OK;
}

int sc_set_stream(sc_ctx *ctx, void *stream) {
  if (!ctx) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  API_END
}

int sc_set_state(sc_ctx *ctx, const double *delta, const double *a_internal) {
  if (!ctx || !delta) return SC_ERR_ARG;
  API_BEGIN
  const size_t nn = ctx->nn0(), nd = (size_t)2 * ctx->S.nc * nn;
  CUDA_TRY(cudaMemcpyAsync(ctx->xstate.p, delta, nd * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  if (a_internal)
    CUDA_TRY(cudaMemcpyAsync(ctx->xstate.p + nd, a_internal, 2 * nn * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  else
    CUDA_TRY(cudaMemsetAsync(ctx->xstate.p + nd, 0, 2 * nn * sizeof(double), ctx->stream));
  if (!ctx->has_vp()) CUDA_TRY(cudaMemsetAsync(ctx->xstate.p + nd, 0, 2 * nn * sizeof(double), ctx->stream));
  k_mask<<<grid1(nd, 256), 256, 0, ctx->stream>>>(2 * ctx->S.nc, nn, ctx->dom.p, ctx->xstate.p);
  check_launch(ctx);
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_set_state_device(sc_ctx *ctx, const double *d_delta, const double *d_a) {
  if (!ctx || !d_delta) return SC_ERR_ARG;
  API_BEGIN
  const size_t nn = ctx->nn0(), nd = (size_t)2 * ctx->S.nc * nn;
  CUDA_TRY(cudaMemcpyAsync(ctx->xstate.p, d_delta, nd * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_a && ctx->has_vp())
    CUDA_TRY(cudaMemcpyAsync(ctx->xstate.p + nd, d_a, 2 * nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  else
    CUDA_TRY(cudaMemsetAsync(ctx->xstate.p + nd, 0, 2 * nn * sizeof(double), ctx->stream));
  k_mask<<<grid1(nd, 256), 256, 0, ctx->stream>>>(2 * ctx->S.nc, nn, ctx->dom.p, ctx->xstate.p);
  check_launch(ctx);
  API_END
}

int sc_get_state(sc_ctx *ctx, double *delta, double *a_internal) {
  if (!ctx) return SC_ERR_ARG;
  API_BEGIN
  const size_t nn = ctx->nn0(), nd = (size_t)2 * ctx->S.nc * nn;
  if (delta) CUDA_TRY(cudaMemcpyAsync(delta, ctx->xstate.p, nd * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (a_internal)
    CUDA_TRY(cudaMemcpyAsync(a_internal, ctx->xstate.p + nd, 2 * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_get_state_device(sc_ctx *ctx, double *d_delta, double *d_a) {
  if (!ctx) return SC_ERR_ARG;
  API_BEGIN
  const size_t nn = ctx->nn0(), nd = (size_t)2 * ctx->S.nc * nn;
  if (d_delta) CUDA_TRY(cudaMemcpyAsync(d_delta, ctx->xstate.p, nd * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  if (d_a) CUDA_TRY(cudaMemcpyAsync(d_a, ctx->xstate.p + nd, 2 * nn * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  API_END
}

int sc_compute(sc_ctx *ctx, int n, double *residual, int *converged) {
  if (!ctx || n < 0) return SC_ERR_ARG;
  if (ctx->S.keldysh) {
    ctx->err = "sc_compute: an LDOS context iterates with sc_ldos_iterate";
    return SC_ERR_STATE;
  }
  API_BEGIN
  if (stream_captured(ctx)) {
    // The caller records the iterations into its own CUDA graph.  Only a
    // steady iteration (the form that replays unchanged) may be recorded, and
    // nothing is read back: a capture allows no synchronisation.
    const bool steady = !ctx->first_compute && ctx->boundary_initialized &&
                        (ctx->frames_zeroed || ctx->chunks.size() > 1) && !ctx->profiling && !ctx->batch_member;
    if (!steady)
      throw EngineError(SC_ERR_STATE,
                        "sc_compute under stream capture: run one iteration outside the capture first "
                        "(profiling off, not a batch grain)");
    for (int i = 0; i < n; ++i) {
      if (ctx->mode == SC_MODE_FP64) compute_iteration<double>(ctx);
      else compute_iteration<float>(ctx);
    }
    return SC_OK;
  }
  for (int i = 0; i < n; ++i) {
    if (ctx->mode == SC_MODE_FP64) compute_iteration<double>(ctx);
    else compute_iteration<float>(ctx);
  }
  read_scalars(ctx);
  const Scalars &s = ctx->host_scalars;
  if (residual) *residual = s.residual;
  if (converged)
    *converged = (s.residual < ctx->S.conv_crit && s.conv_op && s.conv_j && s.conv_fe) ? 1 : 0;
  API_END
}

int sc_burn_in(sc_ctx *ctx, int n, double *residual, int *converged) {
  if (!ctx || n < 0) return SC_ERR_ARG;
  API_BEGIN
  if (stream_captured(ctx))
    throw EngineError(SC_ERR_STATE, "sc_burn_in: not available under stream capture (it reads the residual back)");
  ctx->drop_graph();
  for (int i = 0; i < n; ++i) {
    if (ctx->mode == SC_MODE_FP64) burn_in_once<double>(ctx);
    else burn_in_once<float>(ctx);
  }
  read_scalars(ctx);
  if (residual) *residual = ctx->host_scalars.res_bc;
  if (converged) *converged = ctx->host_scalars.res_bc < ctx->S.conv_crit ? 1 : 0;
  API_END
}

int sc_get_results(sc_ctx *ctx, double *delta_new, double *j, double *a_new) {
  if (!ctx) return SC_ERR_ARG;
  API_BEGIN
  const size_t nn = ctx->nn0(), nd = (size_t)2 * ctx->S.nc * nn;
  if (delta_new) CUDA_TRY(cudaMemcpyAsync(delta_new, ctx->gstate.p, nd * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (j) CUDA_TRY(cudaMemcpyAsync(j, ctx->j_real.p, 2 * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (a_new) CUDA_TRY(cudaMemcpyAsync(a_new, ctx->gstate.p + nd, 2 * nn * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_ldos_dims(const sc_ctx *ctx, int *n_energies, int *per_block, int *n_blocks) {
  if (!ctx || !ctx->S.keldysh) return SC_ERR_ARG;
  if (n_energies) *n_energies = (int)ctx->S.ldos_energies.size();
  if (per_block) *per_block = ctx->S.ldos_block;
  if (n_blocks) *n_blocks = ctx->S.ldos_n_blocks;
  return SC_OK;
}

int sc_ldos_energies(const sc_ctx *ctx, double *energies, double *broadening) {
  if (!ctx || !ctx->S.keldysh) return SC_ERR_ARG;
  if (energies)
    std::memcpy(energies, ctx->S.ldos_energies.data(), ctx->S.ldos_energies.size() * sizeof(double));
  if (broadening) *broadening = ctx->S.ldos_broadening;
  return SC_OK;
}

int sc_ldos_begin_block(sc_ctx *ctx, int block) {
  if (!ctx || !ctx->S.keldysh) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  ldos_begin_block(ctx, block);
  API_END
}

int sc_ldos_iterate(sc_ctx *ctx, int n, double *residual, int *converged) {
  if (!ctx || !ctx->S.keldysh || n < 0) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  for (int i = 0; i < n; ++i) {
    if (ctx->mode == SC_MODE_FP64) ldos_once<double>(ctx);
    else ldos_once<float>(ctx);
  }
  read_scalars(ctx);
  const Scalars &s = ctx->host_scalars;
  if (residual) *residual = s.residual;
  if (converged) *converged = s.residual < ctx->S.conv_crit ? 1 : 0;
  API_END
}

int sc_ldos_run(sc_ctx *ctx, int burnin, int it_min, int it_max, int *converged, int *iterations) {
  if (!ctx || !ctx->S.keldysh) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  // runPostprocess (run_simulation.h:44-104) with runIterations
  // (run_iteration.h:75-130); "until converged" loops stop after 100000.
  const int cap = 100000;
  const double crit = ctx->S.conv_crit;
  int total = 0;
  bool all = true;
  for (int b = 0; b < ctx->S.ldos_n_blocks; ++b) {
    ldos_begin_block(ctx, b);
    if (!(burnin == 0)) {
      for (int i = 1; i <= cap; ++i) {
        if (ctx->mode == SC_MODE_FP64) burn_in_once<double>(ctx);
        else burn_in_once<float>(ctx);
        read_scalars(ctx);
        ++total;
        const bool conv = ctx->host_scalars.res_bc < crit;
        if ((conv && i >= burnin) || (burnin >= 0 && i >= burnin)) break;
      }
    }
    bool conv = false;
    if (!(it_min == 0 && it_max == 0)) {
      for (int i = 1; i <= cap; ++i) {
        if (ctx->mode == SC_MODE_FP64) ldos_once<double>(ctx);
        else ldos_once<float>(ctx);
        read_scalars(ctx);
        ++total;
        conv = ctx->host_scalars.residual < crit;
        if ((conv && i >= it_min) || (it_max >= 0 && i >= it_max)) break;
      }
    }
    if (!conv) {
      all = false;
      break;
    }
  }
  if (converged) *converged = all ? 1 : 0;
  if (iterations) *iterations = total;
  API_END
}

int sc_ldos_get(sc_ctx *ctx, double *ldos) {
  if (!ctx || !ctx->S.keldysh || !ldos) return SC_ERR_ARG;
  API_BEGIN
  const size_t n = ctx->S.ldos_energies.size() * ctx->nn0();
  CUDA_TRY(cudaMemcpyAsync(ldos, ctx->ldos_all.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_ldos_get_device(sc_ctx *ctx, double *d_ldos) {
  if (!ctx || !ctx->S.keldysh || !d_ldos) return SC_ERR_ARG;
  API_BEGIN
  const size_t n = ctx->S.ldos_energies.size() * ctx->nn0();
  CUDA_TRY(cudaMemcpyAsync(d_ldos, ctx->ldos_all.p, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_get_scalars(sc_ctx *ctx, double *out) {
  if (!ctx || !out) return SC_ERR_ARG;
  API_BEGIN
  read_scalars(ctx);
  const Scalars &s = ctx->host_scalars;
  const double v[11] = {s.fe, s.fe_area, s.fe_mag, s.fe_mag_area, s.res_op, s.res_j,
                        s.res_fe, s.res_vp, s.res_bc, s.residual, (double)ctx->S.n_grain};
  std::memcpy(out, v, sizeof(v));
  API_END
}

int sc_get_frame_labels(const sc_ctx *ctx, int angle, signed char *labels, int *box) {
  if (!ctx || angle < 0 || angle >= ctx->S.n_angles) return SC_ERR_ARG;
  const size_t nn1 = (size_t)ctx->S.n1 * ctx->S.n1;
  if (labels) std::memcpy(labels, &ctx->S.labels[(size_t)angle * nn1], nn1);
  if (box) {
    box[0] = ctx->S.x0[angle];
    box[1] = ctx->S.x1[angle];
    box[2] = ctx->S.y0[angle];
    box[3] = ctx->S.y1[angle];
  }
  return SC_OK;
}

int sc_get_domain(const sc_ctx *ctx, signed char *domain) {
  if (!ctx || !domain) return SC_ERR_ARG;
  std::memcpy(domain, ctx->S.domain_ref.data(), ctx->S.domain_ref.size());
  return SC_OK;
}

int sc_boundary_sizes(const sc_ctx *ctx, int *sizes) {
  if (!ctx || !sizes) return SC_ERR_ARG;
  for (int w = 0; w < 4; ++w) sizes[w] = ctx->n_bnd(w);
  return SC_OK;
}

int sc_sweep_plan(const sc_ctx *ctx, int *n_chunks, int *paired) {
  if (!ctx) return SC_ERR_ARG;
  if (n_chunks) *n_chunks = (int)ctx->chunks.size();
  if (paired) *paired = ctx->pair > 0 ? 1 : 0;
  return SC_OK;
}

int sc_get_boundary(sc_ctx *ctx, int which, double *values) {
  if (!ctx || which < 0 || which > 3 || !values) return SC_ERR_ARG;
  API_BEGIN
  const size_t n = (size_t)ctx->n_bnd(which) * ctx->S.ne;
  if (n) {
    if (ctx->mode == SC_MODE_FP64) {
      CUDA_TRY(cudaMemcpyAsync(values, ctx->bnd_ptr(which), n * 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    } else {
      double *tmp = nullptr;
      CUDA_TRY(cudaMallocAsync(&tmp, n * 2 * sizeof(double), ctx->stream));
      k_to_interleaved<float><<<grid1(n, 256), 256, 0, ctx->stream>>>(n, (const Cx<float> *)ctx->bnd_ptr(which), tmp);
      check_launch(ctx);
      CUDA_TRY(cudaMemcpyAsync(values, tmp, n * 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
      CUDA_TRY(cudaFreeAsync(tmp, ctx->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_set_boundary(sc_ctx *ctx, int which, const double *values) {
  if (!ctx || which < 0 || which > 3 || !values) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  const size_t n = (size_t)ctx->n_bnd(which) * ctx->S.ne;
  if (n) {
    if (ctx->mode == SC_MODE_FP64) {
      CUDA_TRY(cudaMemcpyAsync(ctx->bnd_ptr(which), values, n * 2 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    } else {
      double *tmp = nullptr;
      CUDA_TRY(cudaMallocAsync(&tmp, n * 2 * sizeof(double), ctx->stream));
      CUDA_TRY(cudaMemcpyAsync(tmp, values, n * 2 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      k_from_interleaved<float><<<grid1(n, 256), 256, 0, ctx->stream>>>(n, tmp, (Cx<float> *)ctx->bnd_ptr(which));
      check_launch(ctx);
      CUDA_TRY(cudaFreeAsync(tmp, ctx->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  ctx->boundary_initialized = true;
  API_END
}

int sc_boundary_initial(sc_ctx *ctx) {
  if (!ctx) return SC_ERR_ARG;
  ctx->drop_graph();
  API_BEGIN
  if (ctx->mode == SC_MODE_FP64) boundary_initial<double>(ctx);
  else boundary_initial<float>(ctx);
  launch_scalars_b(ctx, 1, 0, 0);
  read_scalars(ctx);
  API_END
}

int sc_angle_greens(sc_ctx *ctx, int angle, double *f, double *g_re, double *i_re) {
  if (!ctx || angle < 0 || angle >= ctx->S.n_angles) return SC_ERR_ARG;
  ctx->drop_graph();
  if (ctx->S.keldysh) {
    ctx->err = "sc_angle_greens: not available on an LDOS context";
    return SC_ERR_STATE;
  }
  API_BEGIN
  const HostSetup &S = ctx->S;
  // The trajectory columns of this angle, swept on their own (unpaired) with
  // the frame written to slot 0.
  std::vector<int4> cols;
  int kmax = 0;
  for (int x = S.x0[angle]; x <= S.x1[angle]; ++x) {
    const int lo = S.col_lo[(size_t)angle * S.n1 + x], hi = S.col_hi[(size_t)angle * S.n1 + x];
    if (lo < 0) continue;
    cols.push_back(make_int4(angle, x, lo, hi));
    kmax = std::max(kmax, hi - lo + 1);
  }
  const size_t nn1 = (size_t)S.n1 * S.n1;
  extend_reference(ctx);
  ctx->frames_zeroed = false;  // slot 0 now holds this angle
  CUDA_TRY(cudaMemsetAsync(ctx->w_fr, 0, nn1 * ctx->frame_rec(), ctx->stream));
  if (!cols.empty()) {
    // Place the columns at the front of the item array (restored below).
    std::vector<int4> saved(cols.size());
    CUDA_TRY(cudaMemcpy(saved.data(), ctx->items.p, cols.size() * sizeof(int4), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(ctx->items.p, cols.data(), cols.size() * sizeof(int4), cudaMemcpyHostToDevice));
    Chunk one{angle, angle + 1, 0, (int)cols.size(), kmax};
    if (ctx->mode == SC_MODE_FP64) launch_sweep<double>(ctx, one, 0);
    else launch_sweep<float>(ctx, one, 0);
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    CUDA_TRY(cudaMemcpy(ctx->items.p, saved.data(), cols.size() * sizeof(int4), cudaMemcpyHostToDevice));
  }
  std::vector<double2> hf(nn1), hg(nn1);
  if (ctx->frame_rec() == 2 * sizeof(double2)) {
    std::vector<double2> rec(2 * nn1);
    CUDA_TRY(cudaMemcpyAsync(rec.data(), ctx->w_fr, nn1 * ctx->frame_rec(), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < nn1; ++i) {
      hf[i] = rec[2 * i];
      hg[i] = rec[2 * i + 1];
    }
  } else {
    std::vector<float2> rec(2 * nn1);
    CUDA_TRY(cudaMemcpyAsync(rec.data(), ctx->w_fr, nn1 * ctx->frame_rec(), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (size_t i = 0; i < nn1; ++i) {
      hf[i] = make_double2(rec[2 * i].x, rec[2 * i].y);
      hg[i] = make_double2(rec[2 * i + 1].x, rec[2 * i + 1].y);
    }
  }
  for (size_t i = 0; i < nn1; ++i) {
    if (f) {
      f[i] = hf[i].x;
      f[nn1 + i] = hf[i].y;
    }
    if (g_re) g_re[i] = hg[i].x;
    if (i_re) i_re[i] = hg[i].y;
  }
  API_END
}

int sc_poisson(sc_ctx *ctx, const double *j, double *a_out) {
  if (!ctx || !j || !a_out) return SC_ERR_ARG;
  ctx->drop_graph();
  if (!ctx->has_vp() || ctx->S.keldysh) {
    ctx->err = "sc_poisson: the configuration has no finite penetration depth (or is an LDOS context)";
    return SC_ERR_STATE;
  }
  API_BEGIN
  const size_t nn2 = 2 * ctx->nn0();
  // Subtract the mean on the host input (ComputeVectorPotential::subtractMean).
  std::vector<double> s(j, j + nn2);
  for (int d = 0; d < 2; ++d) {
    double sum = 0.0;
    for (size_t i = 0; i < nn2 / 2; ++i) sum += s[d * nn2 / 2 + i];
    const double mean = sum / (double)ctx->S.n_grain;
    for (size_t i = 0; i < nn2 / 2; ++i) s[d * nn2 / 2 + i] -= mean;
  }
  CUDA_TRY(cudaMemcpyAsync(ctx->tmp_io.p, s.data(), nn2 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  double *out = ctx->tmp_io.p + nn2;
  poisson(ctx, ctx->tmp_io.p, out, 0);
  CUDA_TRY(cudaMemcpyAsync(a_out, out, nn2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  API_END
}

int sc_measure_fma_peak(int precision, double *flops_per_second) {
  sc_ctx *ctx = nullptr;
  if (!flops_per_second || (precision != 32 && precision != 64)) return SC_ERR_ARG;
  API_BEGIN
  int dev = 0, sms = 0;
  CUDA_TRY(cudaGetDevice(&dev));
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  void *out = nullptr;
  CUDA_TRY(cudaMalloc(&out, 16));
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  const int blocks = sms * 8, iters = 4096;
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    CUDA_TRY(cudaEventRecord(e0));
    if (precision == 64) k_fma_peak<double><<<blocks, 256>>>(iters, 0.999999, 1e-7, (double *)out);
    else k_fma_peak<float><<<blocks, 256>>>(iters, 0.999999f, 1e-7f, (float *)out);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaEventRecord(e1));
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  *flops_per_second = 2.0 * 8.0 * (double)iters * blocks * 256.0 / (best * 1e-3);
  API_END
}

int sc_profile(sc_ctx *ctx, int enable) {
  if (!ctx) return SC_ERR_ARG;
  ctx->drop_graph();
  ctx->profiling = enable != 0;
  return SC_OK;
}

int sc_profile_read(sc_ctx *ctx, int kernel, double *total_ms, long long *launches) {
  if (!ctx || kernel < 0 || kernel > 4) return SC_ERR_ARG;
  API_BEGIN
  CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  double t = 0.0;
  for (auto &pr : ctx->prof[kernel]) {
    float ms = 0.0f;
    CUDA_TRY(cudaEventElapsedTime(&ms, pr.first, pr.second));
    t += ms;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
  }
  if (total_ms) *total_ms = t;
  if (launches) *launches = (long long)ctx->prof[kernel].size();
  ctx->prof[kernel].clear();
  API_END
}

int sc_launch_count(const sc_ctx *ctx, long long *count) {
  if (!ctx || !count) return SC_ERR_ARG;
  *count = ctx->launches;
  return SC_OK;
}

}  // extern "C"

// ===================================================================== batch
// Many independent grains advanced together (one iteration of every active
// grain per call).  Each grain is an ordinary context (its own state, static
// tables, accelerator and convergence) whose sweep work buffers come from one
// pool.  Grains are packed into waves that fit the pool; the Riccati sweep of a
// wave is ONE persistent launch over the columns of all its grains, longest
// columns first.  After the first iteration the whole iteration (all waves and
// all per-grain kernels) is captured once in a CUDA graph and replayed until a
// grain converges and leaves the active set.
struct sc_batch {
  std::vector<sc_ctx *> grains;
  int mode = SC_MODE_FP64;
  cudaStream_t stream = nullptr;
  std::string err;
  int ept_max = 4;     // at most this many energies per thread; each grain the fewest threads per column that allow it
  int minb = 1;        // resident-block variant of the persistent sweep
  int n_sm = 148;
  std::vector<char> active;
  std::vector<int> iterations;
  std::vector<int> grain_state;  // SC_GRAIN_*: running, converged, at its iteration cap, diverged
  DevArray<double> pool;
  size_t pool_bytes = 0;
  // One launch of the persistent sweep: the work units and SweepArgs<R> of
  // the grains that take part (an energy pass of each grain with energies left).
  struct Pass {
    DevArray<int2> units;
    int n_units = 0;
    int ept = 0;  // largest energies per thread among the pass's grains
    DevArray<unsigned char> args;
  };
  struct Wave {
    std::vector<int> grains;
    std::vector<std::unique_ptr<Pass>> passes;  // energy passes, swept one after another
  };
  std::vector<std::unique_ptr<Wave>> waves;
  DevArray<int> counters;
  DevArray<const Scalars *> scalar_src;
  DevArray<Scalars> scalars;  // gathered [grain] after every iteration
  std::vector<Scalars> host_scalars;
  bool use_graph = true;
  cudaGraphExec_t exec = nullptr;
  bool graph_dirty = true;
  long long launches = 0;           // batch-level launches issued eagerly or at capture
  long long graph_launches = 0;     // kernel launches in the captured iteration
  long long replayed_launches = 0;  // launches executed through graph replays
  long long captured_launches = 0;  // launches recorded into graphs (not run at capture)
  // Side streams for the grains' own kernels, forked from and joined back
  // into the batch stream around every phase (graph branches once captured).
  static constexpr int K_SIDE = 8;
  cudaStream_t side[K_SIDE] = {};
  cudaEvent_t ev_fork = nullptr, ev_join[K_SIDE] = {};
  ~sc_batch() {
    if (exec) cudaGraphExecDestroy(exec);
    for (int k = 0; k < K_SIDE; ++k) {
      if (side[k]) cudaStreamDestroy(side[k]);
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (sc_ctx *c : grains) delete c;
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

__global__ void k_gather_scalars(int n, const Scalars *const *src, Scalars *dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = *src[i];
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }
size_t grain_footprint(const sc_ctx *c) {
  return align256(c->need_scratch) + align256(c->need_scratch2) + align256(c->need_frame);
}

// Packs the active grains into waves (largest first, first fit) and points
// every grain's work buffers into the pool at its wave offset.
template <typename R>
void batch_plan(sc_batch *b) {
  std::vector<int> order;
  for (int g = 0; g < (int)b->grains.size(); ++g)
    if (b->active[g]) order.push_back(g);
  std::sort(order.begin(), order.end(), [&](int x, int y) {
    return grain_footprint(b->grains[x]) > grain_footprint(b->grains[y]);
  });
  std::vector<size_t> used;
  std::vector<std::vector<int>> members;
  for (int g : order) {
    const size_t f = grain_footprint(b->grains[g]);
    size_t w = 0;
    while (w < used.size() && used[w] + f > b->pool_bytes) ++w;
    if (w == used.size()) {
      used.push_back(0);
      members.emplace_back();
    }
    sc_ctx *c = b->grains[g];
    char *base = (char *)b->pool.p + used[w];
    c->frames_zeroed = false;  // new place in the pool
    c->w_scratch = (double *)base;
    base += align256(c->need_scratch);
    c->w_scratch2 = (double *)base;
    base += align256(c->need_scratch2);
    c->w_fr = (double *)base;
    used[w] += f;
    members[w].push_back(g);
  }
  b->waves.clear();

  for (auto &m : members) {
    auto wv = std::make_unique<sc_batch::Wave>();
    wv->grains = m;
    int n_passes = 1;
    for (int k = 0; k < (int)m.size(); ++k) {
      sc_ctx *c = b->grains[m[k]];
      const int ne = c->e_pass;  // energies per pass: all of them up to 64, else 32
      c->log_groups = 0;
      while (((ne + (1 << c->log_groups) - 1) >> c->log_groups) > b->ept_max && c->log_groups < 3)
        c->log_groups++;
      c->groups = 1 << c->log_groups;
      c->ept = (ne + c->groups - 1) / c->groups;
      n_passes = std::max(n_passes, (c->S.ne + ne - 1) / ne);
    }
    for (int p = 0; p < n_passes; ++p) {
      wv->passes.push_back(std::make_unique<sc_batch::Pass>());
      sc_batch::Pass &ps = *wv->passes.back();
      std::vector<SweepArgs<R>> args;
      std::vector<std::pair<int, int2>> keyed;  // (column length, unit)
      for (int k = 0; k < (int)m.size(); ++k) {
        sc_ctx *c = b->grains[m[k]];
        const int e = p * c->e_pass;
        if (e >= c->S.ne) continue;
        const int per_warp = 32 >> c->log_groups;
        const Chunk &ch = c->chunks[0];
        SweepArgs<R> A = sweep_args<R>(c, &ch, 0);
        if (c->e_pass < c->S.ne) {
          A.ne = std::min(c->e_pass, c->S.ne - e);
          A.accumulate = e > 0;
          A.e_re += e;
          A.e_im += e;
          A.res += e;
          A.bin_g += e;
          A.bout_g += e;
          A.bin_gt += e;
          A.bout_gt += e;
        }
        const int slot = (int)args.size();
        args.push_back(A);
        ps.ept = std::max(ps.ept, c->ept);
        const int n = ch.item_end - ch.item_begin;
        const int4 *items = c->h_items.data() + ch.item_begin;
        for (int i = 0; i < n; i += per_warp) {
          int len = 0;
          for (int j = i; j < std::min(n, i + per_warp); ++j) len = std::max(len, items[j].w - items[j].z + 1);
          keyed.push_back({len, make_int2(slot, i)});
        }
      }
      std::stable_sort(keyed.begin(), keyed.end(), [](const auto &x, const auto &y) { return x.first > y.first; });
      std::vector<int2> units;
      for (auto &kv : keyed) units.push_back(kv.second);
      ps.n_units = (int)units.size();
      ps.units.upload(units, b->stream);
      std::vector<unsigned char> raw(args.size() * sizeof(SweepArgs<R>));
      std::memcpy(raw.data(), args.data(), raw.size());
      ps.args.upload(raw, b->stream);
    }
    b->waves.push_back(std::move(wv));
  }
  b->counters.alloc(std::max<size_t>(1, b->waves.size()));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  b->graph_dirty = true;
}

template <typename R>
void launch_batch_sweep(sc_batch *b, sc_batch::Wave &w, int wi) {
  int *counter = b->counters.p + wi;
  for (auto &pp : w.passes) {
    sc_batch::Pass &ps = *pp;
    const SweepArgs<R> *args = (const SweepArgs<R> *)ps.args.p;
    CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), b->stream));
    const int ept = ps.ept;
    auto run = [&](auto kernel) {
      int per_sm = 1;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, 0);
      const int blocks = std::max(1, per_sm) * b->n_sm;
      kernel<<<blocks, 128, 0, b->stream>>>(args, ps.units.p, ps.n_units, counter);
    };
    // Mixed precision with at most four energies per thread in the pass: the
    // packed FP32 sweep (each grain's count rounded up to even; a cap of one
    // energy per thread keeps the scalar form, which that mapping is for).
    static const bool no_packed = std::getenv("SCB_NO_PACKED") != nullptr;
    bool packed = false;
    if constexpr (std::is_same<R, float>::value) packed = !no_packed && b->ept_max >= 2 && ept <= 4;
    if constexpr (std::is_same<R, float>::value) {
      if (packed) {
        if (ept <= 2 && b->minb == 6) run(k_sweep_batch<R, 2, 6, true>);
        else if (ept <= 2) run(k_sweep_batch<R, 2, 4, true>);
        else if (b->minb == 4) run(k_sweep_batch<R, 4, 4, true>);
        else if (b->minb == 3) run(k_sweep_batch<R, 4, 3, true>);
        else run(k_sweep_batch<R, 4, 1, true>);
      }
    }
    if (packed) {
    } else if (ept <= 2 && b->minb == 6) {
      run(k_sweep_batch<R, 2, 6>);
    } else if (ept <= 2 && b->minb == 4) {
      run(k_sweep_batch<R, 2, 4>);
    } else if (ept <= 4) {
      if (b->minb == 4) run(k_sweep_batch<R, 4, 4>);
      else if (b->minb == 3) run(k_sweep_batch<R, 4, 3>);
      else run(k_sweep_batch<R, 4, 1>);
    } else if (ept <= 8) {
      run(k_sweep_batch<R, 8, 1>);
    } else {
      run(k_sweep_batch<R, 16, 1>);
    }
    b->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw EngineError(SC_ERR_CUDA, std::string("batch sweep launch: ") + cudaGetErrorString(e));
  }
}

void batch_fork(sc_batch *b) {
  CUDA_TRY(cudaEventRecord(b->ev_fork, b->stream));
  for (int k = 0; k < sc_batch::K_SIDE; ++k) CUDA_TRY(cudaStreamWaitEvent(b->side[k], b->ev_fork, 0));
}
void batch_join(sc_batch *b) {
  for (int k = 0; k < sc_batch::K_SIDE; ++k) {
    CUDA_TRY(cudaEventRecord(b->ev_join[k], b->side[k]));
    CUDA_TRY(cudaStreamWaitEvent(b->stream, b->ev_join[k], 0));
  }
}
// Grain g's kernels go to side stream (rank of g among the active grains) mod K.
void batch_assign_streams(sc_batch *b, bool to_side) {
  int k = 0;
  for (size_t g = 0; g < b->grains.size(); ++g)
    b->grains[g]->stream = (to_side && b->active[g]) ? b->side[(k++) % sc_batch::K_SIDE] : b->stream;
}

// The sweeps of all waves (with the per-grain frame fields before and the
// frame rotation after each wave's launch).
template <typename R>
void batch_sweeps(sc_batch *b) {
  const int nw = (int)b->waves.size();
  batch_assign_streams(b, true);
  for (int wi = 0; wi < nw; ++wi) {
    sc_batch::Wave &w = *b->waves[wi];
    batch_fork(b);
    for (int g : w.grains) {
      sc_ctx *c = b->grains[g];
      const Chunk &ch = c->chunks[0];
      const size_t nn1 = (size_t)c->S.n1 * c->S.n1;
      const int nslots = chunk_slots(c, ch);
      if (!c->frames_zeroed) {
        CUDA_TRY(cudaMemsetAsync(c->w_fr, 0, (size_t)nslots * nn1 * c->frame_rec(), c->stream));
        c->frames_zeroed = true;
      }
      launch_frame_fields<R>(c, ch, sweep_args<R>(c, &ch, 0));
    }
    batch_join(b);
    launch_batch_sweep<R>(b, w, wi);
    batch_fork(b);
    for (int g : w.grains) frame_to_reference<R>(b->grains[g], b->grains[g]->chunks[0]);
    batch_join(b);
  }
  batch_assign_streams(b, false);
}

template <typename R>
void batch_iteration(sc_batch *b) {
  batch_assign_streams(b, true);
  batch_fork(b);
  for (size_t g = 0; g < b->grains.size(); ++g)
    if (b->active[g]) compute_pre<R>(b->grains[g]);
  batch_join(b);
  batch_sweeps<R>(b);
  batch_assign_streams(b, true);
  batch_fork(b);
  for (size_t g = 0; g < b->grains.size(); ++g)
    if (b->active[g]) compute_post<R>(b->grains[g]);
  batch_join(b);
  batch_assign_streams(b, false);
  k_gather_scalars<<<grid1(b->grains.size(), 128), 128, 0, b->stream>>>((int)b->grains.size(), b->scalar_src.p,
                                                                          b->scalars.p);
  b->launches++;
}

template <typename R>
void batch_step(sc_batch *b) {
  bool first = false;
  for (size_t g = 0; g < b->grains.size(); ++g)
    if (b->active[g] && (b->grains[g]->first_compute || !b->grains[g]->boundary_initialized)) first = true;
  if (!b->use_graph || first) {
    batch_iteration<R>(b);  // first iterations differ (no accelerator step, initial boundary)
  } else {
    if (b->graph_dirty || !b->exec) {
      if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
      }
      cudaGraph_t graph = nullptr;
      const long long launches0 = b->launches;
      long long grain_launches0 = 0;
      for (const sc_ctx *c : b->grains) grain_launches0 += c->launches;
      CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      try {
        batch_iteration<R>(b);
      } catch (...) {
        cudaStreamEndCapture(b->stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
      }
      CUDA_TRY(cudaStreamEndCapture(b->stream, &graph));
      b->graph_launches = b->launches - launches0;
      for (const sc_ctx *c : b->grains) b->graph_launches += c->launches;
      b->graph_launches -= grain_launches0;
      b->captured_launches += b->graph_launches;  // counted at capture, run by replays
      const cudaError_t e = cudaGraphInstantiate(&b->exec, graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) throw EngineError(SC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
      b->graph_dirty = false;
    }
    CUDA_TRY(cudaGraphLaunch(b->exec, b->stream));
    b->replayed_launches += b->graph_launches;
  }
  CUDA_TRY(cudaMemcpyAsync(b->host_scalars.data(), b->scalars.p, b->grains.size() * sizeof(Scalars),
                           cudaMemcpyDeviceToHost, b->stream));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  bool changed = false;
  for (size_t g = 0; g < b->grains.size(); ++g) {
    if (!b->active[g]) continue;
    sc_ctx *c = b->grains[g];
    c->host_scalars = b->host_scalars[g];
    b->iterations[g]++;
    const Scalars &s = c->host_scalars;
    // A grain whose iteration produced a non-finite residual or free energy
    // has diverged: it is frozen (leaves the batch with its last state, for
    // inspection) and reported, and the other grains go on unchanged.
    if (!std::isfinite(s.residual) || !std::isfinite(s.fe)) {
      b->active[g] = 0;
      b->grain_state[g] = SC_GRAIN_DIVERGED;
      changed = true;
      continue;
    }
    const bool conv = s.residual < c->S.conv_crit && s.conv_op && s.conv_j && s.conv_fe;
    const bool done = (conv && b->iterations[g] >= c->S.it_min) ||
                      (c->S.it_max >= 0 && b->iterations[g] >= c->S.it_max);
    if (done) {
      b->active[g] = 0;
      b->grain_state[g] = conv ? SC_GRAIN_CONVERGED : SC_GRAIN_AT_CAP;
      changed = true;
    }
  }
  if (changed) batch_plan<R>(b);
}

int batch_fail(sc_batch *b, const EngineError &e) {
  if (b) b->err = e.msg;
  else g_create_error = e.msg;
  return e.code;
}

}  // namespace

extern "C" {

int sc_batch_create(const char *const *configs, int n, int mode, sc_batch **out) {
  if (!configs || n < 1 || !out || (mode != SC_MODE_FP64 && mode != SC_MODE_MIXED)) {
    g_create_error = "sc_batch_create: bad argument";
    return SC_ERR_ARG;
  }
  *out = nullptr;
  sc_batch *b = new sc_batch();
  b->mode = mode;
  try {
    CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    for (int k = 0; k < sc_batch::K_SIDE; ++k) {
      CUDA_TRY(cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking));
      CUDA_TRY(cudaEventCreateWithFlags(&b->ev_join[k], cudaEventDisableTiming));
    }
    CUDA_TRY(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
    int dev = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, dev));
    for (int i = 0; i < n; ++i) {
      if (!configs[i]) throw EngineError(SC_ERR_ARG, "null configuration");
      sc_ctx *c = new sc_ctx();
      b->grains.push_back(c);
      c->mode = mode;
      c->batch_member = true;
    }
    // Host set-up of the grains in parallel (pure host work).
    std::vector<std::string> errs(n);
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < n; ++i) errs[i] = build_setup(configs[i], b->grains[i]->S);
    for (int i = 0; i < n; ++i) {
      sc_ctx *c = b->grains[i];
      const std::string &e = errs[i];
      if (!e.empty()) throw EngineError(SC_ERR_ARG, "grain " + std::to_string(i) + ": " + e);
      if (c->S.nc > MAX_COMP) throw EngineError(SC_ERR_ARG, "at most 4 order-parameter components");
      c->device = dev;
      c->stream = b->stream;
      upload_static(c);
    }
    // Pool: every grain's own footprint must fit; the pool holds as many
    // grains per wave as 60% of the free memory allows.
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    size_t budget = (size_t)(0.6 * (double)free_b);
    if (const char *env = std::getenv("SCB_BATCH_POOL_MB")) budget = (size_t)(std::atof(env) * 1048576.0);
    size_t total = 0, largest = 0;
    for (sc_ctx *c : b->grains) {
      total += grain_footprint(c);
      largest = std::max(largest, grain_footprint(c));
    }
    if (largest > budget) throw EngineError(SC_ERR_SIZE, "a grain's sweep buffers exceed the device memory budget");
    b->pool_bytes = std::min(total, budget);
    b->pool.alloc(b->pool_bytes / sizeof(double) + 1);
    b->active.assign(n, 1);
    b->iterations.assign(n, 0);
    b->grain_state.assign(n, SC_GRAIN_RUNNING);
    std::vector<const Scalars *> src(n);
    for (int i = 0; i < n; ++i) src[i] = b->grains[i]->scalars.p;
    b->scalar_src.upload(src, b->stream);
    b->scalars.alloc(n);
    b->host_scalars.resize(n);
    // Threads per column, per grain: the fewest that keep at most four
    // energies per thread (mixed precision: the packed FP32 sweep).
    b->ept_max = 4;
    b->minb = 4;
    if (mode == SC_MODE_FP64) batch_plan<double>(b);
    else batch_plan<float>(b);
  } catch (const EngineError &e) {
    g_create_error = e.msg;
    delete b;
    return e.code;
  } catch (const std::exception &e) {
    g_create_error = e.what();
    delete b;
    return SC_ERR_ARG;
  }
  *out = b;
  return SC_OK;
}

int sc_batch_destroy(sc_batch *b) {
  if (!b) return SC_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  delete b;
  return SC_OK;
}

const char *sc_batch_last_error(const sc_batch *b) { return b ? b->err.c_str() : g_create_error.c_str(); }

int sc_batch_size(const sc_batch *b, int *n) {
  if (!b || !n) return SC_ERR_ARG;
  *n = (int)b->grains.size();
  return SC_OK;
}

int sc_batch_grain(sc_batch *b, int i, sc_ctx **ctx) {
  if (!b || !ctx || i < 0 || i >= (int)b->grains.size()) return SC_ERR_ARG;
  *ctx = b->grains[i];
  return SC_OK;
}

int sc_batch_compute(sc_batch *b, int n, int *n_active) {
  if (!b || n < 0) return SC_ERR_ARG;
  try {
    for (int i = 0; i < n; ++i) {
      bool any = false;
      for (char a : b->active) any = any || a;
      if (!any) break;
      if (b->mode == SC_MODE_FP64) batch_step<double>(b);
      else batch_step<float>(b);
    }
    if (n_active) {
      int k = 0;
      for (char a : b->active) k += a;
      *n_active = k;
    }
  } catch (const EngineError &e) {
    return batch_fail(b, e);
  }
  return SC_OK;
}

int sc_batch_status(const sc_batch *b, int *active, int *iterations, double *residual) {
  if (!b) return SC_ERR_ARG;
  for (size_t g = 0; g < b->grains.size(); ++g) {
    if (active) active[g] = b->active[g];
    if (iterations) iterations[g] = b->iterations[g];
    if (residual) residual[g] = b->grains[g]->host_scalars.residual;
  }
  return SC_OK;
}

int sc_batch_grain_state(const sc_batch *b, int *state) {
  if (!b || !state) return SC_ERR_ARG;
  for (size_t g = 0; g < b->grains.size(); ++g) state[g] = b->grain_state[g];
  return SC_OK;
}

int sc_batch_set_graph(sc_batch *b, int enable) {
  if (!b) return SC_ERR_ARG;
  b->use_graph = enable != 0;
  b->graph_dirty = true;
  return SC_OK;
}

int sc_batch_config(sc_batch *b, int energies_per_thread, int minb) {
  const int e = energies_per_thread;
  if (!b || !(e == 1 || e == 2 || e == 4 || e == 8 || e == 16) || (minb != 1 && minb != 3 && minb != 4 && minb != 6))
    return SC_ERR_ARG;
  int ne_max = 1;
  for (sc_ctx *c : b->grains) ne_max = std::max(ne_max, c->S.ne);
  if ((ne_max + 7) / 8 > 16) return SC_ERR_ARG;
  try {
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    b->ept_max = e;
    b->minb = minb;
    if (b->mode == SC_MODE_FP64) batch_plan<double>(b);
    else batch_plan<float>(b);
  } catch (const EngineError &e) {
    return batch_fail(b, e);
  }
  return SC_OK;
}

int sc_batch_get_config(const sc_batch *b, int *energies_per_thread, int *minb, int *n_waves) {
  if (!b) return SC_ERR_ARG;
  if (energies_per_thread) *energies_per_thread = b->ept_max;
  if (minb) *minb = b->minb;
  if (n_waves) *n_waves = (int)b->waves.size();
  return SC_OK;
}

// Times the sweeps of all waves for the current configuration (no state
// changes: the sweeps rewrite the same outgoing boundary values and frames).
int sc_batch_time_sweeps(sc_batch *b, int repeats, double *ms) {
  if (!b || repeats < 1 || !ms) return SC_ERR_ARG;
  try {
    for (size_t g = 0; g < b->grains.size(); ++g)
      if (b->active[g] && !b->grains[g]->boundary_initialized)
        throw EngineError(SC_ERR_STATE, "sc_batch_time_sweeps: run one iteration first");
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0, b->stream));
    for (int r = 0; r < repeats; ++r) {
      if (b->mode == SC_MODE_FP64) batch_sweeps<double>(b);
      else batch_sweeps<float>(b);
    }
    CUDA_TRY(cudaEventRecord(e1, b->stream));
    CUDA_TRY(cudaEventSynchronize(e1));
    float t = 0.0f;
    cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = (double)t / repeats;
  } catch (const EngineError &e) {
    return batch_fail(b, e);
  }
  return SC_OK;
}

int sc_batch_launch_count(const sc_batch *b, long long *count) {
  if (!b || !count) return SC_ERR_ARG;
  long long k = b->launches + b->replayed_launches - b->captured_launches;
  for (const sc_ctx *c : b->grains) k += c->launches;
  *count = k;
  return SC_OK;
}

}  // extern "C"

extern "C" {

// Autotuner of the persistent batch sweep: tries the mappings of trajectory
// columns to threads (at most 1, 2, 4 or 8 energies per thread, each grain
// taking the fewest threads per column that allow it, up to 8) with the
// resident-block variants that fit them (registers capped at 80, 128 or 255
// per thread), times the sweeps of all waves for each on the current state,
// keeps the fastest and returns it.
int sc_batch_autotune(sc_batch *b, int *energies_per_thread, int *minb, double *best_ms) {
  if (!b) return SC_ERR_ARG;
  const int cand[][2] = {{1, 4}, {2, 4}, {2, 6}, {4, 3}, {4, 4}, {4, 1}, {8, 1}};
  int best_e = b->ept_max, best_mb = b->minb;
  double best = 1e300;
  for (const auto &cd : cand) {
    int st = sc_batch_config(b, cd[0], cd[1]);
    if (st != SC_OK) return st;
    double ms = 0.0;
    st = sc_batch_time_sweeps(b, 1, &ms);  // warm-up
    if (st == SC_OK) st = sc_batch_time_sweeps(b, 2, &ms);
    if (st != SC_OK) return st;
    if (ms < best) {
      best = ms;
      best_e = cd[0];
      best_mb = cd[1];
    }
  }
  const int st = sc_batch_config(b, best_e, best_mb);
  if (st != SC_OK) return st;
  if (energies_per_thread) *energies_per_thread = best_e;
  if (minb) *minb = best_mb;
  if (best_ms) *best_ms = best;
  return SC_OK;
}

}  // extern "C"

#include "adjoint.cuh"
