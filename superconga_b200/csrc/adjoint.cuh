// Reverse-mode derivatives of one frozen-boundary evaluation of the
// self-consistency map (included at the end of engine.cu; FP64 contexts).
//
// The functional is
//   L(Delta, A, b) = w_omega * Omega + sum_r (beta_x(r) j_x(r) + beta_y(r) j_y(r)),
// with Omega the free energy of ComputeFreeEnergy (ComputeFreeEnergy.h:281-414)
// and j the current of ComputeCurrent (ComputeCurrent.h:175-222), both from
// one pass of Riccati sweeps over every angle with the incoming boundary
// values held fixed (IntegrationIteratorOzaki.h:302-404 without the boundary
// update).  b is the external field B_ext = pi Phi / area of the gauge
// (RiccatiSolver.h:137-139).
//
// L is linear in the frame sums Re I and Re g of every angle, so the
// derivative starts from seeds on the frame lattice: the transposes of the
// rotation back (insertRotatedGridAdditive) and of the frame extension
// (extendValuesAtBoundary) applied to the reference-grid weights.  The adjoint
// sweep then runs, per trajectory column, the two Riccati recursions forward
// with gamma and gammaTilde checkpointed every ADJ_K sites, and integrates the
// adjoint recursions in reverse, recomputing each ADJ_K-site segment from its
// checkpoint.  Complex sensitivities are carried as G = dL/dRe z + i dL/dIm z:
// G_z = conj(f'(z)) G_w for holomorphic w = f(z), G_z = k conj(G_w) for
// w = k conj(z).  The frame-lattice sensitivities of the rotated order
// parameter and of the Doppler shift are finally scattered back through the
// transposed bilinear lookups onto the reference grid.

namespace {

constexpr int ADJ_K = 16;  // checkpoint interval in trajectory sites

struct AdjArgs {
  SweepArgs<double> S;
  Cx<double> *ck_gt, *ck_g;  // [segment][energy][item] state entering each segment
  int *ck_nin_gt, *ck_nin_g; // [segment][item] entry counters entering each segment
  const double2 *seed;       // [slot][n1*n1] (seed of Re I, seed of Re g)
  double2 *grad_d;           // [slot][n1*n1] dL/dDelta_frame
  double *grad_e;            // [slot][n1*n1] dL/d(Doppler shift)
};

__device__ __forceinline__ Cx<double> cadd(Cx<double> a, Cx<double> b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx<double> cconj(Cx<double> a) { return {a.re, -a.im}; }
__device__ __forceinline__ Cx<double> cscale(Cx<double> a, double s) { return {a.re * s, a.im * s}; }
__device__ __forceinline__ Cx<double> cinv(Cx<double> a) {
  const double n = 1.0 / (a.re * a.re + a.im * a.im);
  return {a.re * n, -a.im * n};
}

// Reverse mode of riccati_step<double> (same intermediates): given gw for g1,
// returns the sensitivities of g0, of the step's order parameter D and of the
// real part of the step's energy.
__device__ __forceinline__ void riccati_step_adj(double dre, double dim, double ere, double eim,
                                                 Cx<double> g0, double h, Cx<double> gw,
                                                 Cx<double> &gg0, Cx<double> &gD, double &ge) {
  typedef Cx<double> C;
  const double q = 0.25 * h;
  const C a{q * dim, q * dre};
  const C ihe{-h * eim, h * ere};
  const C ag = cmul(a, g0);
  const C b{2.0 * ag.re + ihe.re - 1.0, 2.0 * ag.im + ihe.im};
  const C t{ag.re + ihe.re + 1.0, ag.im + ihe.im};
  const C tg = cmul(t, g0);
  const C c{tg.re - h * dim, tg.im + h * dre};
  const C bb = cmul(b, b), ac = cmul(a, c);
  const C s = csqrt_dev<double>(bb.re - 4.0 * ac.re, bb.im - 4.0 * ac.im);
  const C den{s.re - b.re, s.im - b.im};
  const C rden = cinv(den);
  const C g1 = cmul(cscale(c, 2.0), rden);
  // g1 = 2 c / den
  C Gc = cmul(cconj(cscale(rden, 2.0)), gw);
  const C Gden = cmul(cconj(cscale(cmul(g1, rden), -1.0)), gw);
  // den = s - b
  C Gb = cscale(Gden, -1.0);
  // s = sqrt(disc)
  const C Gdisc = cmul(cconj(cscale(cinv(s), 0.5)), Gden);
  // disc = b^2 - 4 a c
  Gb = cadd(Gb, cmul(cconj(cscale(b, 2.0)), Gdisc));
  C Ga = cmul(cconj(cscale(c, -4.0)), Gdisc);
  Gc = cadd(Gc, cmul(cconj(cscale(a, -4.0)), Gdisc));
  // c = t g0 + i h D
  const C Gt = cmul(cconj(g0), Gc);
  gg0 = cmul(cconj(t), Gc);
  // t = a g0 + i h e + 1;  b = 2 a g0 + i h e - 1
  const C Gag = cadd(Gt, cscale(Gb, 2.0));
  const C Gihe = cadd(Gt, Gb);
  Ga = cadd(Ga, cmul(cconj(g0), Gag));
  gg0 = cadd(gg0, cmul(cconj(a), Gag));
  // i h e: G_e = -i h G
  ge = h * Gihe.im;
  // i h D: G_D = -i h G
  gD = C{h * Gc.im, -h * Gc.re};
  // a = (i h / 4) conj(D): G_D += (i h / 4) conj(G_a)
  gD = cadd(gD, C{q * Ga.im, q * Ga.re});
}

__device__ __forceinline__ void fields_at(const SweepArgs<double> &A, size_t ni, int item, int r,
                                          double &f0, double &f1, double &f2) {
  (void)ni;
  const double4 v = ((const double4 *)A.scratch2)[rec_index(A, A.log_groups, item, r)];
  f0 = v.x;
  f1 = v.y;
  f2 = v.z;
}

// The adjoint of one trajectory column for the EMAX energies of thread g.
template <int EMAX>
__device__ void adjoint_column(const AdjArgs &J, const double *s_res, int item, int g, unsigned gmask) {
  typedef Cx<double> C;
  const SweepArgs<double> &A = J.S;
  const int4 it = A.items[item];
  const int a = it.x, x = it.y, lo = it.z, hi = it.w;
  const int n1 = A.n1, ne = A.ne, len = hi - lo + 1;
  const size_t nn1 = (size_t)n1 * n1, ni = (size_t)A.n_items;
  const uint8_t *lab = A.labels + (size_t)a * nn1;
  const double h = A.ang[a].hs;
  const int e0 = g * A.ept;
  int ecount = ne - e0;
  if (ecount > A.ept) ecount = A.ept;
  if (ecount < 0) ecount = 0;
  double eim[EMAX], rr[EMAX];
#pragma unroll
  for (int j = 0; j < EMAX; ++j) {
    eim[j] = (j < ecount) ? A.e_im[e0 + j] : 1.0;
    rr[j] = (j < ecount) ? s_res[e0 + j] : 0.0;
  }
  const size_t ax = (size_t)a * n1 + x;
  const int in_g = A.idx_in_g[ax], in_gt = A.idx_in_gt[ax];
  const size_t slot = (size_t)(a - A.slot_base) * nn1;
  const int nseg = (len + ADJ_K - 1) / ADJ_K;
  auto ck = [&](Cx<double> *base, int seg, int j) -> Cx<double> & {
    return base[((size_t)seg * ne + e0 + j) * ni + item];
  };

  // -------------------------------------------- primal passes, checkpoints --
  C coh[EMAX];
  {  // gammaTilde down
    int nin = 0;
    double p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = C{0, 0};
    for (int r = len - 1; r >= 0; --r) {
      const int seg = r / ADJ_K;
      if (r == len - 1 || r % ADJ_K == ADJ_K - 1) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) ck(J.ck_gt, seg, j) = coh[j];
        if (g == 0) J.ck_nin_gt[(size_t)seg * ni + item] = nin;
      }
      double f0, f1, f2;
      fields_at(A, ni, item, r, f0, f1, f2);
      const double dre = -f0, dim = f1, es = f2;
      const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
      if (l == 0) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j) coh[j] = C{0, 0};
      } else if (l == 3) {
        const double st = A.dist_in_gt[in_gt + nin] * h;
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount)
            coh[j] = riccati_step<double>(dre, dim, es, eim[j], ((const C *)A.bin_gt)[(size_t)(in_gt + nin) * A.ne_stride + e0 + j], st);
        ++nin;
      } else {
        const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) coh[j] = riccati_step<double>(mre, mim, mes, eim[j], coh[j], h);
      }
      p0 = dre;
      p1 = dim;
      p2 = es;
    }
  }
  {  // gamma up
    int nin = 0;
    double p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
    for (int j = 0; j < EMAX; ++j) coh[j] = C{0, 0};
    for (int r = 0; r < len; ++r) {
      if (r % ADJ_K == 0) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) ck(J.ck_g, r / ADJ_K, j) = coh[j];
        if (g == 0) J.ck_nin_g[(size_t)(r / ADJ_K) * ni + item] = nin;
      }
      double dre, dim, es;
      fields_at(A, ni, item, r, dre, dim, es);
      const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
      if (l == 0) {
#pragma unroll
        for (int j = 0; j < EMAX; ++j) coh[j] = C{0, 0};
      } else if (l == 2) {
        const double st = A.dist_in_g[in_g + nin] * h;
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount)
            coh[j] = riccati_step<double>(dre, dim, es, eim[j], ((const C *)A.bin_g)[(size_t)(in_g + nin) * A.ne_stride + e0 + j], st);
        ++nin;
      } else {
        const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
#pragma unroll
        for (int j = 0; j < EMAX; ++j)
          if (j < ecount) coh[j] = riccati_step<double>(mre, mim, mes, eim[j], coh[j], h);
      }
      p0 = dre;
      p1 = dim;
      p2 = es;
    }
  }
  __syncwarp(gmask);

  // Segment replays: gamma (up) and gammaTilde (down) of rows [rb, rt].
  C Lg[ADJ_K][EMAX], Lgt[ADJ_K][EMAX];
  auto replay = [&](int seg, int rb, int rt) {
    {  // gamma up from the segment's checkpoint
      int nin = J.ck_nin_g[(size_t)seg * ni + item];
      double p0 = 0, p1 = 0, p2 = 0;
      if (rb > 0) fields_at(A, ni, item, rb - 1, p0, p1, p2);
      C cc[EMAX];
#pragma unroll
      for (int j = 0; j < EMAX; ++j) cc[j] = (j < ecount) ? ck(J.ck_g, seg, j) : C{0, 0};
      for (int r = rb; r <= rt; ++r) {
        double dre, dim, es;
        fields_at(A, ni, item, r, dre, dim, es);
        const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
        if (l == 0) {
#pragma unroll
          for (int j = 0; j < EMAX; ++j) cc[j] = C{0, 0};
        } else if (l == 2) {
          const double st = A.dist_in_g[in_g + nin] * h;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount)
              cc[j] = riccati_step<double>(dre, dim, es, eim[j], ((const C *)A.bin_g)[(size_t)(in_g + nin) * A.ne_stride + e0 + j], st);
          ++nin;
        } else {
          const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) cc[j] = riccati_step<double>(mre, mim, mes, eim[j], cc[j], h);
        }
#pragma unroll
        for (int j = 0; j < EMAX; ++j) Lg[r - rb][j] = cc[j];
        p0 = dre;
        p1 = dim;
        p2 = es;
      }
    }
    {  // gammaTilde down from the segment's checkpoint
      int nin = J.ck_nin_gt[(size_t)seg * ni + item];
      double p0 = 0, p1 = 0, p2 = 0;
      if (rt < len - 1) {
        fields_at(A, ni, item, rt + 1, p0, p1, p2);
        p0 = -p0;
      }
      C cc[EMAX];
#pragma unroll
      for (int j = 0; j < EMAX; ++j) cc[j] = (j < ecount) ? ck(J.ck_gt, seg, j) : C{0, 0};
      for (int r = rt; r >= rb; --r) {
        double f0, f1, f2;
        fields_at(A, ni, item, r, f0, f1, f2);
        const double dre = -f0, dim = f1, es = f2;
        const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
        if (l == 0) {
#pragma unroll
          for (int j = 0; j < EMAX; ++j) cc[j] = C{0, 0};
        } else if (l == 3) {
          const double st = A.dist_in_gt[in_gt + nin] * h;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount)
              cc[j] = riccati_step<double>(dre, dim, es, eim[j], ((const C *)A.bin_gt)[(size_t)(in_gt + nin) * A.ne_stride + e0 + j], st);
          ++nin;
        } else {
          const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) cc[j] = riccati_step<double>(mre, mim, mes, eim[j], cc[j], h);
        }
#pragma unroll
        for (int j = 0; j < EMAX; ++j) Lgt[r - rb][j] = cc[j];
        p0 = dre;
        p1 = dim;
        p2 = es;
      }
    }
  };

  // Local seeds of one site: the sensitivity of the loss to gamma (or
  // gammaTilde) through Re I and Re g at that site.
  //   Re I = -sum r [Im(conj(D) g) - Im(D gt)],  Re g = Im((1 - g gt)/(1 + g gt)).
  auto gp_of = [&](C gm, C gtl, double sg, double r) -> C {
    const C p = cmul(gm, gtl);
    const C onep{1.0 + p.re, p.im};
    const C inv = cinv(onep);
    const C dq = cscale(cmul(inv, inv), -2.0);          // dQ/dp
    const C GQ{0.0, sg * r};                             // Re g = Im Q
    return cmul(cconj(dq), GQ);                          // G_p
  };

  // ------------------------------------------ adjoint of gamma, top-down --
  // Row r's order-parameter and shift sensitivities collect the step at r
  // (half, midpoint) and the step at r + 1 (the other half, carried in pend).
  {
    C lam[EMAX];
#pragma unroll
    for (int j = 0; j < EMAX; ++j) lam[j] = C{0, 0};
    C pendD{0, 0};
    double pendE = 0.0;
    for (int seg = nseg - 1; seg >= 0; --seg) {
      const int rb = seg * ADJ_K, rt = min(rb + ADJ_K, len) - 1;
      replay(seg, rb, rt);
      for (int r = rt; r >= rb; --r) {
        double dre, dim, es;
        fields_at(A, ni, item, r, dre, dim, es);
        const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
        const size_t site = (size_t)(lo + r) * n1 + x;
        C ownD{0, 0};
        double ownE = 0.0;
        C pendNext{0, 0};
        double pendNextE = 0.0;
        if (l != 0) {
          const double2 sd = J.seed[slot + site];
          const C D{dre, dim};
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) {
              const C gm = Lg[r - rb][j], gtl = Lgt[r - rb][j];
              // Re I: G_g = -sI r i D ; direct G_D = sI r i (g + conj(gt))
              const C iD{-D.im, D.re};
              lam[j] = cadd(lam[j], cscale(iD, -sd.x * rr[j]));
              const C s1 = cadd(gm, cconj(gtl));
              ownD = cadd(ownD, cscale(C{-s1.im, s1.re}, sd.x * rr[j]));
              // Re g: G_g = conj(gt) G_p
              lam[j] = cadd(lam[j], cmul(cconj(gtl), gp_of(gm, gtl, sd.y, rr[j])));
            }
          if (l == 2) {
            int nin = J.ck_nin_g[(size_t)seg * ni + item];
            for (int r2 = rb; r2 < r; ++r2) nin += lab[(size_t)(lo + r2) * n1 + x] == 2;
            const double st = A.dist_in_g[in_g + nin] * h;
#pragma unroll
            for (int j = 0; j < EMAX; ++j)
              if (j < ecount) {
                C gg0, gD;
                double ge;
                riccati_step_adj(dre, dim, es, eim[j], ((const C *)A.bin_g)[(size_t)(in_g + nin) * A.ne_stride + e0 + j], st,
                                 lam[j], gg0, gD, ge);
                ownD = cadd(ownD, gD);
                ownE += ge;
                lam[j] = C{0, 0};
              }
          } else {
            double p0 = 0, p1 = 0, p2 = 0;
            if (r > 0) fields_at(A, ni, item, r - 1, p0, p1, p2);
            const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
            C nD{0, 0};
            double nE = 0.0;
#pragma unroll
            for (int j = 0; j < EMAX; ++j)
              if (j < ecount) {
                const C gin = (r - 1 >= rb) ? Lg[r - 1 - rb][j] : ck(J.ck_g, seg, j);
                C gg0, gD;
                double ge;
                riccati_step_adj(mre, mim, mes, eim[j], gin, h, lam[j], gg0, gD, ge);
                nD = cadd(nD, gD);
                nE += ge;
                lam[j] = gg0;
              }
            ownD = cadd(ownD, cscale(nD, 0.5));
            ownE += 0.5 * nE;
            if (r > 0) {
              pendNext = cscale(nD, 0.5);
              pendNextE = 0.5 * nE;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < EMAX; ++j) lam[j] = C{0, 0};
        }
        ownD = cadd(ownD, pendD);
        ownE += pendE;
        pendD = pendNext;
        pendE = pendNextE;
        if (A.groups > 1) {
          group_sum(ownD.re, A.groups, gmask);
          group_sum(ownD.im, A.groups, gmask);
          group_sum(ownE, A.groups, gmask);
        }
        if (g == 0) {
          if (A.accumulate) {  // a later energy pass adds to the earlier ones
            const double2 o = J.grad_d[slot + site];
            J.grad_d[slot + site] = make_double2(o.x + ownD.re, o.y + ownD.im);
            J.grad_e[slot + site] += ownE;
          } else {
            J.grad_d[slot + site] = make_double2(ownD.re, ownD.im);
            J.grad_e[slot + site] = ownE;
          }
        }
      }
    }
  }
  __syncwarp(gmask);

  // ---------------------------------------- adjoint of gammaTilde, bottom-up --
  {
    C lam[EMAX];
#pragma unroll
    for (int j = 0; j < EMAX; ++j) lam[j] = C{0, 0};
    C pendD{0, 0};
    double pendE = 0.0;
    for (int seg = 0; seg < nseg; ++seg) {
      const int rb = seg * ADJ_K, rt = min(rb + ADJ_K, len) - 1;
      replay(seg, rb, rt);
      for (int r = rb; r <= rt; ++r) {
        double f0, f1, f2;
        fields_at(A, ni, item, r, f0, f1, f2);
        const double dre = -f0, dim = f1, es = f2;  // gammaTilde's order parameter -conj(Delta)
        const uint8_t l = lab[(size_t)(lo + r) * n1 + x];
        const size_t site = (size_t)(lo + r) * n1 + x;
        C ownT{0, 0};  // sensitivity to -conj(Delta) at this row
        double ownE = 0.0;
        C pendNext{0, 0};
        double pendNextE = 0.0;
        if (l != 0) {
          const double2 sd = J.seed[slot + site];
          const C D{f0, f1};
#pragma unroll
          for (int j = 0; j < EMAX; ++j)
            if (j < ecount) {
              const C gm = Lg[r - rb][j], gtl = Lgt[r - rb][j];
              // Re I: G_gt = sI r i conj(D)
              const C icD{D.im, D.re};
              lam[j] = cadd(lam[j], cscale(icD, sd.x * rr[j]));
              // Re g: G_gt = conj(g) G_p
              lam[j] = cadd(lam[j], cmul(cconj(gm), gp_of(gm, gtl, sd.y, rr[j])));
            }
          if (l == 3) {
            int nin = J.ck_nin_gt[(size_t)seg * ni + item];
            for (int rr2 = rt; rr2 > r; --rr2) nin += lab[(size_t)(lo + rr2) * n1 + x] == 3;
            const double st = A.dist_in_gt[in_gt + nin] * h;
#pragma unroll
            for (int j = 0; j < EMAX; ++j)
              if (j < ecount) {
                C gg0, gD;
                double ge;
                riccati_step_adj(dre, dim, es, eim[j], ((const C *)A.bin_gt)[(size_t)(in_gt + nin) * A.ne_stride + e0 + j], st,
                                 lam[j], gg0, gD, ge);
                ownT = cadd(ownT, gD);
                ownE += ge;
                lam[j] = C{0, 0};
              }
          } else {
            double p0 = 0, p1 = 0, p2 = 0;
            if (r < len - 1) {
              fields_at(A, ni, item, r + 1, p0, p1, p2);
              p0 = -p0;
            }
            const double mre = (dre + p0) * 0.5, mim = (dim + p1) * 0.5, mes = (es + p2) * 0.5;
            C nD{0, 0};
            double nE = 0.0;
#pragma unroll
            for (int j = 0; j < EMAX; ++j)
              if (j < ecount) {
                const C gin = (r + 1 <= rt) ? Lgt[r + 1 - rb][j] : ck(J.ck_gt, seg, j);
                C gg0, gD;
                double ge;
                riccati_step_adj(mre, mim, mes, eim[j], gin, h, lam[j], gg0, gD, ge);
                nD = cadd(nD, gD);
                nE += ge;
                lam[j] = gg0;
              }
            ownT = cadd(ownT, cscale(nD, 0.5));
            ownE += 0.5 * nE;
            if (r < len - 1) {
              pendNext = cscale(nD, 0.5);
              pendNextE = 0.5 * nE;
            }
          }
        } else {
#pragma unroll
          for (int j = 0; j < EMAX; ++j) lam[j] = C{0, 0};
        }
        // -conj(Delta) -> Delta: G_Delta = -conj(G)
        C ownD{-ownT.re, ownT.im};
        ownD = cadd(ownD, pendD);
        ownE += pendE;
        pendD = C{-pendNext.re, pendNext.im};
        pendE = pendNextE;
        if (A.groups > 1) {
          group_sum(ownD.re, A.groups, gmask);
          group_sum(ownD.im, A.groups, gmask);
          group_sum(ownE, A.groups, gmask);
        }
        if (g == 0) {
          const double2 o = J.grad_d[slot + site];
          J.grad_d[slot + site] = make_double2(o.x + ownD.re, o.y + ownD.im);
          J.grad_e[slot + site] += ownE;
        }
      }
    }
  }
}

template <int EMAX>
__global__ void __launch_bounds__(128) k_adjoint(const AdjArgs J) {
  __shared__ double s_res[64];
  for (int e = threadIdx.x; e < J.S.ne && e < 64; e += blockDim.x) s_res[e] = J.S.res[e];
  __syncthreads();
  const SweepArgs<double> &A = J.S;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int item = tid >> A.log_groups;
  const int g = tid & (A.groups - 1);
  const int lane = threadIdx.x & 31;
  const unsigned gmask = ((A.groups == 32) ? 0xffffffffu : ((1u << A.groups) - 1u)) << (lane & ~(A.groups - 1));
  if (item >= A.n_items) return;
  adjoint_column<EMAX>(J, s_res, item, g, gmask);
}

// Seeds on the frame lattice of the angles [a_begin, a_end): the transpose of
// the rotation back (k_rotate_back) applied to the reference-grid weights
// alpha (of Re I, already times the integrand factor's partner T h^2 w_omega)
// and beta (of j_x, j_y, already times the current's factor).
__global__ void k_adj_seeds(int n0, int n1, int a_begin, int a_end, const AngleParams *__restrict__ ang,
                            const double *__restrict__ alpha, const double *__restrict__ beta, double2 *seed) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= n0 || y >= n0) return;
  const size_t nn0 = (size_t)n0 * n0, nn1 = (size_t)n1 * n1;
  const size_t i = (size_t)y * n0 + x;
  const double al = alpha[i], bx = beta[i], by = beta[nn0 + i];
  if (al == 0.0 && bx == 0.0 && by == 0.0) return;
  for (int a = a_begin; a < a_end; ++a) {
    const AngleParams &P = ang[a];
    Bilinear b;
    if (!rotated_lookup(x, y, n0, n1, P.cB, P.sB, b)) continue;
    const double vi = al * P.w, vg = bx * P.sx + by * P.sy;
    const double w[4] = {(1.0 - b.xf) * (1.0 - b.yf), b.xf * (1.0 - b.yf), (1.0 - b.xf) * b.yf, b.xf * b.yf};
    const int off[4] = {b.i00, b.i00 + 1, b.i00 + n1, b.i00 + n1 + 1};
    double *s = (double *)(seed + (size_t)(a - a_begin) * nn1);
    for (int k = 0; k < 4; ++k) {
      atomicAdd(s + 2 * (size_t)off[k], w[k] * vi);
      atomicAdd(s + 2 * (size_t)off[k] + 1, w[k] * vg);
    }
  }
}

// Transpose of the frame extension (k_halo): a halo site's seed moves to its
// sources in equal parts.
__global__ void k_adj_halo_t(int n_entries, int entry0, int n1, const int *__restrict__ entry_angle,
                             int slot_base, const int *__restrict__ site, const int *__restrict__ off,
                             const int *__restrict__ src, double2 *seed) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_entries) return;
  const int e = entry0 + k;
  double *s = (double *)(seed + (size_t)(entry_angle[e] - slot_base) * n1 * n1);
  const double2 v = ((double2 *)s)[site[e]];
  ((double2 *)s)[site[e]] = make_double2(0.0, 0.0);
  const int b = off[e], en = off[e + 1];
  const double inv = 1.0 / (double)(en - b);
  for (int i = b; i < en; ++i) {
    atomicAdd(s + 2 * (size_t)src[i], v.x * inv);
    atomicAdd(s + 2 * (size_t)src[i] + 1, v.y * inv);
  }
}

// Frame sensitivities back onto the reference grid: the transposes of the
// bilinear lookups of frame_fields (order parameter, induced vector potential)
// and the derivative of the gauge potential with respect to the field.
__global__ void __launch_bounds__(256) k_adj_fields_t(SweepArgs<double> A, int a_begin, int a_end,
                                                      const double2 *__restrict__ grad_d,
                                                      const double *__restrict__ grad_e, double *g_dext,
                                                      double *g_avec, double *g_b) {
  const int n1 = A.n1, n0 = A.n0;
  const size_t nn1 = (size_t)n1 * n1, nn0 = (size_t)n0 * n0;
  const size_t site = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const int a = a_begin + blockIdx.y;
  double gb = 0.0;
  if (site < nn1 && a < a_end) {
    const AngleParams &P = A.ang[a];
    const int x = (int)(site % n1), y = (int)(site / n1);
    const double2 gd = grad_d[(size_t)(a - a_begin) * nn1 + site];
    const double ge = grad_e[(size_t)(a - a_begin) * nn1 + site];
    Bilinear b;
    if ((gd.x != 0.0 || gd.y != 0.0) && rotated_lookup(x, y, n1, n0, P.cD, P.sD, b)) {
      const double w[4] = {(1.0 - b.xf) * (1.0 - b.yf), b.xf * (1.0 - b.yf), (1.0 - b.xf) * b.yf, b.xf * b.yf};
      const int off[4] = {b.i00, b.i00 + 1, b.i00 + n0, b.i00 + n0 + 1};
      for (int c = 0; c < A.nc; ++c) {
        double *pr = g_dext + (size_t)(2 * c) * nn0, *pi = pr + nn0;
        const double et = P.eta[c];
        for (int k = 0; k < 4; ++k) {
          atomicAdd(pr + off[k], w[k] * et * gd.x);
          atomicAdd(pi + off[k], w[k] * et * gd.y);
        }
      }
    }
    if (ge != 0.0) {  // the shift depends on the field even where it is zero
      const double off = -0.5 * (double)(n1 - 1);
      const double xp = ((double)x + off) * A.h, yp = ((double)y + off) * A.h;
      const double xr = xp * P.cE - yp * P.sE, yr = xp * P.sE + yp * P.cE;
      double ax1 = 0.0, ay1 = 0.0;
      gauge_potential(A.gauge, 1.0, A.area, xr, yr, ax1, ay1);
      gb = ge * A.q * (P.vx * ax1 + P.vy * ay1);
      Bilinear ba;
      if (A.has_vp && rotated_lookup(x, y, n1, n0, P.cA, P.sA, ba)) {
        const double w[4] = {(1.0 - ba.xf) * (1.0 - ba.yf), ba.xf * (1.0 - ba.yf), (1.0 - ba.xf) * ba.yf,
                             ba.xf * ba.yf};
        const int off4[4] = {ba.i00, ba.i00 + 1, ba.i00 + n0, ba.i00 + n0 + 1};
        const double gx = ge * A.q * P.vx * A.lam_scale, gy = ge * A.q * P.vy * A.lam_scale;
        for (int k = 0; k < 4; ++k) {
          atomicAdd(g_avec + off4[k], w[k] * gx);
          atomicAdd(g_avec + nn0 + off4[k], w[k] * gy);
        }
      }
    }
  }
  // block sum of the field sensitivity
  __shared__ double sh[256];
  sh[threadIdx.x] = gb;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0 && sh[0] != 0.0) atomicAdd(g_b, sh[0]);
}

// Transpose of extend_reference: an extension site's sensitivity moves to its
// sources in equal parts.
__global__ void k_adj_rext_t(int n_fields, int nn, int n_sites, const int *__restrict__ site,
                             const int *__restrict__ off, const int *__restrict__ src, double *g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (k >= n_sites || f >= n_fields) return;
  double *gf = g + (size_t)f * nn;
  const double v = gf[site[k]];
  gf[site[k]] = 0.0;
  const int b = off[k], e = off[k + 1];
  const double inv = 1.0 / (double)(e - b);
  for (int i = b; i < e; ++i) atomicAdd(gf + src[i], v * inv);
}

// Explicit terms of the free energy: sum_c |Delta_c|^2 (ln(T/Tc_c) + T sum r/e)
// inside the grain (times h^2 w_omega), and the mask of the order parameter
// (zero outside the grain, OrderParameter.h:180-199).
__global__ void k_adj_explicit(int n0, int nc, const uint8_t *__restrict__ dom, const double *__restrict__ x,
                               const double *__restrict__ coef, double *g) {
  const size_t nn = (size_t)n0 * n0;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  for (int c = 0; c < nc; ++c)
    for (int p = 0; p < 2; ++p) {
      const size_t k = (size_t)(2 * c + p) * nn + i;
      g[k] = dom[i] ? g[k] + 2.0 * coef[c] * x[k] : 0.0;
    }
}

// Magnetic term h^2 w_omega (0.5 / lambda^2) sum B^2 with B the curl of the
// stored vector potential (curl_kernel, GridFunctions_GPU.h:326-352).
__global__ void k_adj_curl_t(int n0, double h, double scale, const double *__restrict__ avec, double *g_avec) {
  const size_t nn = (size_t)n0 * n0;
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const int x = (int)(i % n0), y = (int)(i / n0);
  const int xn = min(x + 1, n0 - 1), xp = max(x - 1, 0);
  const int yn = min(y + 1, n0 - 1), yp = max(y - 1, 0);
  const double *ax = avec, *ay = avec + nn;
  const double dx = (double)(xn - xp), dy = (double)(yn - yp);
  const double bz = ((ay[(size_t)y * n0 + xn] - ay[(size_t)y * n0 + xp]) / dx -
                     (ax[(size_t)yn * n0 + x] - ax[(size_t)yp * n0 + x]) / dy) / h;
  const double gbz = 2.0 * scale * bz / h;
  atomicAdd(g_avec + nn + (size_t)y * n0 + xn, gbz / dx);
  atomicAdd(g_avec + nn + (size_t)y * n0 + xp, -gbz / dx);
  atomicAdd(g_avec + (size_t)yn * n0 + x, -gbz / dy);
  atomicAdd(g_avec + (size_t)yp * n0 + x, gbz / dy);
}

// Frozen-boundary evaluation: g(x), j and the free energy of the current
// state without an accelerator step and without the boundary update.
void evaluate_once(sc_ctx *c) {
  const HostSetup &S = c->S;
  if (!c->boundary_initialized) boundary_initial<double>(c);
  extend_reference(c);
  c->acc_d.zero(c->stream);
  c->acc_j.zero(c->stream);
  c->acc_fe.zero(c->stream);
  run_chunks<double>(c, 0);
  const size_t nn = c->nn0();
  double *delta = c->xstate.p, *avec = c->xstate.p + (size_t)2 * S.nc * nn;
  const double jfactor = (double)(2 * S.charge_sign) * S.temperature;
  k_finalize<<<c->nb_fin, REDUCE_THREADS, 0, c->stream>>>(
      S.n0, S.nc, S.h, jfactor, c->has_vp() ? 1 : 0, c->dom.p, c->coupling.p, c->acc_d.p, c->acc_j.p, c->acc_fe.p,
      delta, avec, c->gstate.p, c->j_real.p, c->partial_fin.p);
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

struct AdjBuffers {
  DevArray<double> ck, grad_e, g_dext, g_avec, g_b, alpha, beta, coef;
  DevArray<int> ck_nin;
};
void AdjDeleter::operator()(AdjBuffers *p) const { delete p; }

void adjoint_run(sc_ctx *c, AdjBuffers &B, double w_omega, const double *beta_host, double *g_delta,
                 double *g_a, double *g_b) {
  const HostSetup &S = c->S;
  const size_t nn = c->nn0();
  const size_t nn1 = (size_t)S.n1 * S.n1;
  // Per-chunk buffers.
  size_t ck_n = 0, nin_n = 0, slots = 0;
  for (const Chunk &ch : c->chunks) {
    const size_t ni = (size_t)(ch.item_end - ch.item_begin);
    const size_t nseg = (size_t)(ch.kmax + ADJ_K - 1) / ADJ_K;
    ck_n = std::max(ck_n, 2 * nseg * S.ne * ni);
    nin_n = std::max(nin_n, 2 * nseg * ni);
    slots = std::max(slots, (size_t)(ch.a_end - ch.a_begin));
  }
  if (B.ck.n < 2 * ck_n) B.ck.alloc(2 * ck_n);  // complex: 2 doubles each
  if (B.ck_nin.n < nin_n) B.ck_nin.alloc(nin_n);
  if (B.grad_e.n < slots * nn1) B.grad_e.alloc(slots * nn1);
  B.g_dext.alloc((size_t)2 * S.nc * nn);
  B.g_avec.alloc(2 * nn);
  B.g_b.alloc(1);
  B.g_dext.zero(c->stream);
  B.g_avec.zero(c->stream);
  B.g_b.zero(c->stream);
  // Reference-grid weights of Re I (free energy) and of the current.
  std::vector<double> alpha(nn), beta(2 * nn, 0.0);
  const double la = S.h * S.h;
  const double jfactor = (double)(2 * S.charge_sign) * S.temperature;
  for (size_t i = 0; i < nn; ++i) alpha[i] = S.domain_ref[i] ? w_omega * la * S.temperature : 0.0;
  if (beta_host)
    for (size_t i = 0; i < 2 * nn; ++i) beta[i] = S.domain_ref[i % nn] ? beta_host[i] * jfactor : 0.0;
  B.alpha.upload(alpha, c->stream);
  B.beta.upload(beta, c->stream);
  extend_reference(c);
  for (const Chunk &ch : c->chunks) {
    const int nslots = ch.a_end - ch.a_begin;
    SweepArgs<double> A = sweep_args<double>(c, &ch, 0);
    if (!A.n_items) continue;
    launch_frame_fields<double>(c, ch, A);
    // The frame-record buffer (two double2 per site and slot) holds both.
    double2 *seed = (double2 *)c->w_fr, *grad_d = seed + (size_t)nslots * nn1;
    c->frames_zeroed = false;  // the frame buffers serve as seed and gradient buffers
    CUDA_TRY(cudaMemsetAsync(seed, 0, (size_t)nslots * nn1 * sizeof(double2), c->stream));
    CUDA_TRY(cudaMemsetAsync(grad_d, 0, (size_t)nslots * nn1 * sizeof(double2), c->stream));
    CUDA_TRY(cudaMemsetAsync(B.grad_e.p, 0, (size_t)nslots * nn1 * sizeof(double), c->stream));
    {
      dim3 blk(32, 8), grid((S.n0 + 31) / 32, (S.n0 + 7) / 8);
      k_adj_seeds<<<grid, blk, 0, c->stream>>>(S.n0, S.n1, ch.a_begin, ch.a_end, c->ang.p, B.alpha.p, B.beta.p, seed);
      check_launch(c);
      const int h0 = S.halo_angle_off[ch.a_begin], h1 = S.halo_angle_off[ch.a_end];
      if (h1 > h0) {
        k_adj_halo_t<<<grid1(h1 - h0, 128), 128, 0, c->stream>>>(h1 - h0, h0, S.n1, c->halo_angle.p, ch.a_begin,
                                                                  c->halo_site.p, c->halo_off.p, c->halo_src.p, seed);
        check_launch(c);
      }
    }
    AdjArgs J{};
    J.S = A;
    const size_t ni = (size_t)A.n_items;
    const size_t nseg = (size_t)(ch.kmax + ADJ_K - 1) / ADJ_K;
    J.ck_gt = (Cx<double> *)B.ck.p;
    J.ck_g = J.ck_gt + nseg * S.ne * ni;
    J.ck_nin_gt = B.ck_nin.p;
    J.ck_nin_g = B.ck_nin.p + nseg * ni;
    J.seed = seed;
    J.grad_d = grad_d;
    J.grad_e = B.grad_e.p;
    const size_t threads = ni * c->groups;
    if (c->ept <= 4 && c->e_pass >= S.ne) {
      k_adjoint<4><<<grid1(threads, 128), 128, 0, c->stream>>>(J);
      check_launch(c);
    } else {
      // Energy passes of four energies per thread, each from its own slice
      // of the boundary values, adding into the gradients of the earlier ones.
      const int pass = 4 * c->groups;
      for (int e = 0; e < S.ne; e += pass) {
        AdjArgs P = J;
        P.S.ne = std::min(pass, S.ne - e);
        P.S.ept = 4;
        P.S.accumulate = e > 0;
        P.S.e_re += e;
        P.S.e_im += e;
        P.S.res += e;
        P.S.bin_g += e;
        P.S.bin_gt += e;
        P.S.bout_g += e;
        P.S.bout_gt += e;
        k_adjoint<4><<<grid1(threads, 128), 128, 0, c->stream>>>(P);
        check_launch(c);
      }
    }
    dim3 gridf(grid1(nn1, 256), nslots);
    k_adj_fields_t<<<gridf, 256, 0, c->stream>>>(A, ch.a_begin, ch.a_end, grad_d, B.grad_e.p, B.g_dext.p,
                                                  B.g_avec.p, B.g_b.p);
    check_launch(c);
  }
  // Reference extension transpose, explicit terms, mask.
  const int ns = (int)S.rext_site.size();
  if (ns) {
    dim3 grid(grid1(ns, 128), 2 * S.nc);
    k_adj_rext_t<<<grid, 128, 0, c->stream>>>(2 * S.nc, (int)nn, ns, c->rext_site.p, c->rext_off.p, c->rext_src.p,
                                               B.g_dext.p);
    check_launch(c);
  }
  double si = 0.0;
  for (int e = 0; e < S.ne; ++e) si += S.residues[e] / S.e_im[e];
  std::vector<double> coef(S.nc);
  for (int k = 0; k < S.nc; ++k) coef[k] = w_omega * la * (std::log(S.temperature / S.tc[k]) + si * S.temperature);
  B.coef.upload(coef, c->stream);
  k_adj_explicit<<<grid1(nn, 256), 256, 0, c->stream>>>(S.n0, S.nc, c->dom.p, c->xstate.p, B.coef.p, B.g_dext.p);
  check_launch(c);
  if (c->has_vp() && w_omega != 0.0) {
    const double scale = w_omega * la * 0.5 / (S.lambda * S.lambda);
    k_adj_curl_t<<<grid1(nn, 256), 256, 0, c->stream>>>(S.n0, S.h, scale, c->xstate.p + (size_t)2 * S.nc * nn,
                                                          B.g_avec.p);
    check_launch(c);
  }
  if (g_delta)
    CUDA_TRY(cudaMemcpyAsync(g_delta, B.g_dext.p, (size_t)2 * S.nc * nn * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
  if (g_a) CUDA_TRY(cudaMemcpyAsync(g_a, B.g_avec.p, 2 * nn * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (g_b) CUDA_TRY(cudaMemcpyAsync(g_b, B.g_b.p, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CUDA_TRY(cudaStreamSynchronize(c->stream));
}

}  // namespace

extern "C" {

int sc_set_external_field(sc_ctx *ctx, double b) {
  if (!ctx || ctx->batch_member) return SC_ERR_ARG;
  ctx->drop_graph();
  ctx->S.flux_quanta = b * ctx->S.area / M_PI;
  return SC_OK;
}

int sc_get_external_field(const sc_ctx *ctx, double *b) {
  if (!ctx || !b) return SC_ERR_ARG;
  *b = M_PI * ctx->S.flux_quanta / ctx->S.area;
  return SC_OK;
}

int sc_evaluate(sc_ctx *ctx, double *free_energy) {
  if (!ctx) return SC_ERR_ARG;
  ctx->drop_graph();
  if (ctx->mode != SC_MODE_FP64 || ctx->S.keldysh || ctx->batch_member) {
    ctx->err = "sc_evaluate: FP64 self-consistency contexts only";
    return SC_ERR_STATE;
  }
  API_BEGIN
  evaluate_once(ctx);
  read_scalars(ctx);
  if (free_energy) *free_energy = ctx->host_scalars.fe;
  API_END
}

int sc_adjoint(sc_ctx *ctx, double w_omega, const double *beta_j, double *g_delta, double *g_a,
               double *g_b) {
  if (!ctx) return SC_ERR_ARG;
  ctx->drop_graph();
  if (ctx->mode != SC_MODE_FP64 || ctx->S.keldysh || ctx->batch_member) {
    ctx->err = "sc_adjoint: FP64 self-consistency contexts only";
    return SC_ERR_STATE;
  }
  if (!ctx->boundary_initialized) {
    ctx->err = "sc_adjoint: the boundary values are not set (run an iteration or sc_boundary_initial first)";
    return SC_ERR_STATE;
  }
  API_BEGIN
  if (!ctx->adj) ctx->adj.reset(new AdjBuffers());
  adjoint_run(ctx, *ctx->adj, w_omega, beta_j, g_delta, g_a, g_b);
  API_END
}

}  // extern "C"
