// Adjoint (vector-Jacobian product) of one whole fused step, for the differentiable path.
//
// The step (app/main.f90:280-355 without compression and sources: v12rhov1/T2rhoe,
// set_global_boundaries, halo_fluidvars, interface_vels, the nine field sweeps x3 -> x1 ->
// x2, rhov12v1, clean_param(1..3), rhoe2T, energy_diffusion) maps the state (ns, vs1, Ts
// and the stale x1 boundary faces of vs1i) to the next state.  gem_step_vjp_dev pulls a
// cotangent of the next state back to the state before the step, on the device:
//
//   forward replay (inputs of every sweep kept):
//     conversions + ghost fill (the standalone kernels of the plain path), interface
//     velocities, then per direction: copy the stage, sweep the copy in place;
//   backward, in reverse:
//     post-sweep conversions/floors and the energy diffusion (k_diffusion_vjp),
//     the x2, (periodic wrap), x1 and x3 sweep adjoints (k_sweep_vjp; the x1 ones also
//     accumulate the interface-velocity cotangent), the x3 and x2 ghost copies, the x1
//     boundary extrapolation/reflection, the interface velocities and the conversions.
//
// Conventions of the differentiable step: cotangents at ghost cells of the step's outputs
// are ignored (the next step overwrites every ghost before reading it), and the state's
// ghost cells get zero cotangent.  Ties of min/max split the cotangent in half and clamps
// pass it at equality, as autograd does.
//
// Included by gem_fluid.cu (one translation unit with the plain path).

namespace gemk {

// faces 1 and lx1+1 of a vs1i face array from the (LSP, lx3, lx2) boundary arrays
__global__ void ka_set_faces(Dims d, const double* __restrict__ lo, const double* __restrict__ hi, double* v1i) {
  const long long ncol = (long long)d.lx2 * d.lx3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncol * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / ncol);
    const long long c = t - s * ncol;
    const int i2 = (int)(c % d.lx2) + 1, i3 = (int)(c / d.lx2) + 1;
    v1i[s * nf1(d) + f1i(d, 1, i2, i3)] = lo[t];
    v1i[s * nf1(d) + f1i(d, d.lx1 + 1, i2, i3)] = hi[t];
  }
}

// Traversal of the ghosted grid by 32-cell chunks of x1 rows (i2, i3 ghosts included): one
// warp per chunk, a lane per cell along the contiguous x1, 32-bit index arithmetic; calls
// body(k, i1, i2, i3, interior) for every cell.
template <class Body>
__device__ __forceinline__ void for_rows(const Dims& d, Body body) {
  const int X1 = d.lx1 + 4, X2 = d.lx2 + 4, X3 = d.lx3 + 4;
  const int nch = (X1 + 31) / 32;
  const int nunit = X2 * X3 * nch;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int u = blockIdx.x * wpb + (threadIdx.x >> 5); u < nunit; u += gridDim.x * wpb) {
    const int r = u / nch, ch = u - r * nch;
    const int i2 = r % X2 - 1, i3 = r / X2 - 1;
    const int i1 = ch * 32 + lane - 1;
    if (i1 > d.lx1 + 2) continue;
    const bool in = i1 >= 1 && i1 <= d.lx1 && i2 >= 1 && i2 <= d.lx2 && i3 >= 1 && i3 <= d.lx3;
    body(gi(d, i1, i2, i3), i1, i2, i3, in);
  }
}

// The same traversal with the species as the slowest coordinate: body(k, i1, i2, i3,
// interior, s) for every cell and species (for per-species work with no coupling).
template <class Body>
__device__ __forceinline__ void for_rows_s(const Dims& d, Body body) {
  const int X1 = d.lx1 + 4, X2 = d.lx2 + 4, X3 = d.lx3 + 4;
  const int nch = (X1 + 31) / 32;
  const int nper = X2 * X3 * nch;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int u = blockIdx.x * wpb + (threadIdx.x >> 5); u < nper * LSP; u += gridDim.x * wpb) {
    const int s = u / nper;
    const int uu = u - s * nper;
    const int r = uu / nch, ch = uu - r * nch;
    const int i2 = r % X2 - 1, i3 = r / X2 - 1;
    const int i1 = ch * 32 + lane - 1;
    if (i1 > d.lx1 + 2) continue;
    const bool in = i1 >= 1 && i1 <= d.lx1 && i2 >= 1 && i2 <= d.lx2 && i3 >= 1 && i3 <= d.lx3;
    body(gi(d, i1, i2, i3), i1, i2, i3, in, s);
  }
}

// Post-sweep forward values the diffusion adjoint needs: n after clean_param(1) (ion floor,
// electrons the ion sum; ghosts 1e-5) and T after rhoe2T + clean_param(3) (ghosts 100).
// F: the swept stage (n | rv | re blocks).
__global__ void ka_post_fwd(GridDev G, const double* __restrict__ F, double* nout, double* Tpre) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const double* re = F + 2 * LSP * ng;
  for_rows(d, [&](long long k, int, int, int, bool in) {
    if (!in) {
      for (int s = 0; s < LSP; ++s) {
        nout[s * ng + k] = MINDENSDIV;
        Tpre[s * ng + k] = 100.0;
      }
      return;
    }
    double ne = 0.0;
    for (int s = 0; s < LSP; ++s) {
      double nv;
      if (s < LSP - 1) {
        nv = fmax_f(F[s * ng + k], MINDENS);
        ne += nv;
      } else {
        nv = ne;
      }
      nout[s * ng + k] = nv;
      const double T = c_gm1kb[s] * re[s * ng + k] / fmax_f(nv, MINDENSDIV);
      Tpre[s * ng + k] = fmax_f(T, 100.0);
    }
  });
}

// The forward step's x2 epilogue (rhov12v1 + clean_param(1) + clean_param(2) null fill +
// rhoe2T + clean_param(3), multifluid.f90:179-233) recomputed from a replay's swept stage F
// (n | rv | re): the same operations in the same order as the fused x2 sweep's epilogue
// (products rounded where that kernel rounds them through shared memory), so the interior
// ns, rv, vs1, Ts written into B are the forward step's bits. Ghost cells get the swept n and
// rv, which k_ghost_epilogue then turns into the forward's ghost values.
__global__ void ka_finish_fwd(GridDev G, const double* __restrict__ F, Blocks B) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const double* fn = F;
  const double* frv = F + LSP * ng;
  const double* fre = F + 2 * LSP * ng;
  for_rows(d, [&](long long k, int i1, int i2, int i3, bool in) {
    if (!in) {
      for (int s = 0; s < LSP - 1; ++s) {
        B.ns(s)[k] = fn[s * ng + k];
        B.rv(s)[k] = frv[s * ng + k];
      }
      return;
    }
    const bool nul = is_null(G, i1, i2, i3);
    double npre = 0.0, chrg = 0.0, npost = 0.0;
    for (int s = 0; s < LSP - 1; ++s) {
      const double n = fn[s * ng + k], r = frv[s * ng + k], e = fre[s * ng + k];
      const double v = r / (c_ms[s] * fmax_f(n, MINDENSDIV));
      npre = npre + n;
      chrg = __dadd_rn(chrg, __dmul_rn(__dmul_rn(n, c_qs[s]), v));
      npost = npost + fmax_f(n, MINDENS);
      double nc = fmax_f(n, MINDENS);
      if (nul) nc = (s == 0) ? MINDENSNULL * 1e-2 : MINDENSNULL;
      double T = fmax_f(c_gm1kb[s] * e / fmax_f(nc, MINDENSDIV), 100.0);
      if (nul) T = 100;
      B.ns(s)[k] = nc;
      B.rv(s)[k] = r;
      B.vs1(s)[k] = nul ? 0.0 : v;
      B.Ts(s)[k] = T;
    }
    const int s = LSP - 1;
    const double ve = mdiv(-1 / fmax_f(npre, MINDENSDIV), QE, YQE) * chrg;
    const double ne = nul ? MINDENSNULL : npost;
    double T = fmax_f(c_gm1kb[s] * fre[s * ng + k] / fmax_f(ne, MINDENSDIV), 100.0);
    if (nul) T = 100;
    B.ns(s)[k] = ne;
    B.vs1(s)[k] = nul ? 0.0 : ve;
    B.Ts(s)[k] = T;
  });
}

// The two boundary faces of every x1 column (the state's lo / hi), read from a face array:
// the inverse of ka_set_faces.
__global__ void ka_get_faces(Dims d, const double* __restrict__ v1i, double* lo, double* hi) {
  const long long ncol = (long long)d.lx2 * d.lx3;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncol * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / ncol);
    const long long c = t - s * ncol;
    const int i2 = (int)(c % d.lx2) + 1, i3 = (int)(c / d.lx2) + 1;
    lo[t] = v1i[s * nf1(d) + f1i(d, 1, i2, i3)];
    hi[t] = v1i[s * nf1(d) + f1i(d, d.lx1 + 1, i2, i3)];
  }
}

// Adjoint of rhov12v1 + clean_param(1) + rhoe2T + clean_param(3) (multifluid.f90:218-233,
// 553-688): from the cotangents of the step's n and v1 outputs (interior), of the diffusion
// input T (TPb) and of the diffusion's n input (NDb), the cotangents of the swept n, rv, re
// (C: n | rv | re blocks; ghost cells 0).
__global__ void __launch_bounds__(256) ka_post_vjp(GridDev G, const double* __restrict__ F,
                                                   const double* __restrict__ nbo, const double* __restrict__ vbo,
                                                   const double* __restrict__ TPb, const double* __restrict__ NDb,
                                                   double* C) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const double* rv = F + LSP * ng;
  const double* re = F + 2 * LSP * ng;
  double* cn = C;
  double* crv = C + LSP * ng;
  double* cre = C + 2 * LSP * ng;
  for_rows(d, [&](long long k, int, int, int, bool in) {
    if (!in) {
      for (int s = 0; s < LSP; ++s) {
        cn[s * ng + k] = 0.0;
        crv[s * ng + k] = 0.0;
        cre[s * ng + k] = 0.0;
      }
      return;
    }
    // sums over the ions: n, the floored n (the electron density), the charge flux
    double nsum = 0.0, ne = 0.0, csum = 0.0;
#pragma unroll 1
    for (int s = 0; s < LSP - 1; ++s) {
      const double n = F[s * ng + k];
      nsum += n;
      ne += fmax_f(n, MINDENS);
      const double v1 = rv[s * ng + k] * c_yms[s] / fmax_f(n, MINDENSDIV);
      csum += n * c_qs[s] * v1;
    }
    // energy: T = max((gamma-1)/kB re / max(n_out, 1e-5), 100), n_out the floored density
    auto energy = [&](int s, double nout) -> double {  // returns the cotangent of n_out
      const double D = fmax_f(nout, MINDENSDIV);
      const double Tr = c_gm1kb[s] * re[s * ng + k] / D;  // as the forward: the floor test
      const double Tb = (Tr >= 100.0) ? TPb[s * ng + k] : 0.0;
      const double TbyD = Tb / D;
      cre[s * ng + k] = TbyD * (c_gm1kb[s]);
      double nb = nbo[s * ng + k] + NDb[s * ng + k];
      if (nout >= MINDENSDIV) nb += -TbyD * Tr;
      return nb;
    };
    const double nbe = energy(LSP - 1, ne);  // electrons: n_out = the ion sum
    cn[(LSP - 1) * ng + k] = 0.0;   // the swept electron density is replaced by the ion sum
    crv[(LSP - 1) * ng + k] = 0.0;  // the electron momentum is not advected
    // rhov12v1: v1 = rv/(ms max(n,1e-5)); ve = -(sum n qs v1)/max(sum n, 1e-5)/qs_e
    const double Nn = fmax_f(nsum, MINDENSDIV);
    const double veb = vbo[(LSP - 1) * ng + k];
    const double csb = veb * (-1 / Nn / c_qs[LSP - 1]);
    const double nsb = (nsum >= MINDENSDIV) ? veb * csum / (Nn * Nn) / c_qs[LSP - 1] : 0.0;
#pragma unroll 1
    for (int s = 0; s < LSP - 1; ++s) {
      const double n = F[s * ng + k];
      const double nb = energy(s, fmax_f(n, MINDENS));
      // clean_param(1): ions max(n, 1e-100), electrons their sum
      double c = (n >= MINDENS) ? nb + nbe : 0.0;
      const double yDv = 1.0 / fmax_f(n, MINDENSDIV);
      const double v1 = rv[s * ng + k] * c_yms[s] * yDv;
      const double v1b = vbo[s * ng + k] + csb * n * c_qs[s];
      c += nsb + csb * c_qs[s] * v1;
      if (n >= MINDENSDIV) c += -v1b * v1 * yDv;
      cn[s * ng + k] = c;
      crv[s * ng + k] = v1b * c_yms[s] * yDv;
    }
  });
}

// Adjoint of the periodic x3 self-wrap (mpihalo.f90:147-151) on n, rv, re: rows 1:lx2,
// every x1.  The ghost layers' cotangents move to their source layers.
__global__ void ka_wrap3_vjp(GridDev G, double* C) {
  const Dims d = G.d;
  const int n1 = d.lx1 + 4;
  const long long nrow = (long long)n1 * d.lx2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrow * 3 * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(t / nrow);  // field-species block
    const long long c = t - f * nrow;
    const int i1 = (int)(c % n1) - 1, i2 = (int)(c / n1) + 1;
    double* p = C + (long long)f * d.ng;
    const int dst[4] = {-1, 0, d.lx3 + 1, d.lx3 + 2};
    const int src[4] = {d.lx3 - 1, d.lx3, 1, 2};
    double gq[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long kd = gi(d, i1, i2, dst[q]);
      gq[q] = p[kd];
      p[kd] = 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) p[gi(d, i1, i2, src[q])] += gq[q];
  }
}

// Adjoint of the edge copies into the two ghost layers of direction DIM (2 or 3) on n, rv,
// re, over every cell of the other two directions (advec.f90:83-132).
template <int DIM>
__global__ void ka_copy_vjp(GridDev G, double* C) {
  const Dims d = G.d;
  const int na = d.lx1 + 4;
  const int nb = (DIM == 2) ? d.lx3 + 4 : d.lx2 + 4;
  const int lx = (DIM == 2) ? d.lx2 : d.lx3;
  const long long nrow = (long long)na * nb;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nrow * 3 * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int f = (int)(t / nrow);
    const long long c = t - f * nrow;
    const int i1 = (int)(c % na) - 1, ib = (int)(c / na) - 1;
    double* p = C + (long long)f * d.ng;
    auto at = [&](int j) { return (DIM == 2) ? gi(d, i1, j, ib) : gi(d, i1, ib, j); };
    const double g0 = p[at(-1)] + p[at(0)];
    const double g1 = p[at(lx + 1)] + p[at(lx + 2)];
    p[at(-1)] = 0.0;
    p[at(0)] = 0.0;
    p[at(lx + 1)] = 0.0;
    p[at(lx + 2)] = 0.0;
    p[at(1)] += g0;
    p[at(lx)] += g1;
  }
}

// Before a sweep adjoint writes the cotangent stage Cn from C: the cells its lines do not
// cover -- the ghost frame of the other two directions, and the species past a field's
// nsp -- keep C's value.
template <int DIM>
__global__ void ka_frame_copy(GridDev G, const double* __restrict__ C, double* Cn) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const int X2 = d.lx2 + 4, X3 = d.lx3 + 4;
  const int nrow = X2 * X3 * 3 * LSP;
  const int lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < nrow; r += gridDim.x * wpb) {
    const int b = r / (X2 * X3);  // field-species block
    const int rr = r - b * (X2 * X3);
    const int i2 = rr % X2 - 1, i3 = rr / X2 - 1;
    const int s = b % LSP, fld = b / LSP;
    const bool in2 = i2 >= 1 && i2 <= d.lx2, in3 = i3 >= 1 && i3 <= d.lx3;
    const bool swept = s < ((fld == 2) ? LSP : LSP - 1);
    // rows whose every cell some line covers (x1 lines), or whose interior x1 cells lines cover
    const bool row_line = (DIM == 1) ? (in2 && in3) : (DIM == 2) ? in3 : in2;
    if (swept && row_line && DIM == 1) continue;
    const long long k0 = (long long)b * ng + gi(d, 0, i2, i3);
    for (int i1 = lane - 1; i1 <= d.lx1 + 2; i1 += 32) {
      const bool in1 = i1 >= 1 && i1 <= d.lx1;
      if (swept && row_line && in1) continue;
      Cn[k0 + i1] = C[k0 + i1];
    }
  }
}

// min(a, b) split of a cotangent: all to the smaller, half each on a tie
__device__ __forceinline__ void min_split(double a, double b, double g, double& ga, double& gb) {
  if (a < b) { ga = g; gb = 0.0; }
  else if (a > b) { ga = 0.0; gb = g; }
  else { ga = 0.5 * g; gb = 0.5 * g; }
}

// Adjoint of the x1 boundary of set_global_boundaries (advec.f90:42-79) on the interior
// x1 rows: density ratio extrapolation, momentum reflected from the stale boundary faces,
// constant-temperature energy.  The ghost
// cotangents of n, rv, re go to the row's cells 1..3 / lx1-2..lx1, to the stale faces
// (lob, hib: (LSP, lx3, lx2)) and to v1 at cells 1 and lx1 (vext: 2 x LSP per row, for the
// conversion adjoint).  One thread per (row, species); the species-0 thread also sums the
// exospheric-temperature cotangent over species.
__global__ void ka_x1bc_vjp(GridDev G, const double* __restrict__ ns, const double* __restrict__ vs1,
                            const double* __restrict__ Ts, const double* __restrict__ lo,
                            const double* __restrict__ hi, double* C, double* vext, double* lob, double* hib,
                            const double* __restrict__ ttb, double* Ttop_bar) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const long long ncol = (long long)d.lx2 * d.lx3;
  const int lx = d.lx1;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < ncol * LSP;
       t += (long long)gridDim.x * blockDim.x) {
    const int s = (int)(t / ncol);
    const long long c = t - s * ncol;
    const int i2 = (int)(c % d.lx2) + 1, i3 = (int)(c / d.lx2) + 1;
    auto at = [&](int i1) { return gi(d, i1, i2, i3); };
    {
      const long long o = (long long)s * ng;
      const double* n = ns + o;
      double* cn = C + o;
      double* crv = C + LSP * ng + o;
      double* cre = C + 2 * LSP * ng + o;
      const double ms = c_ms[s];
      double v1b1 = 0.0, v1bl = 0.0;
      // ---- bottom
      {
        const double n1 = n[at(1)], n2 = n[at(2)], n3 = n[at(3)];
        const double cl = n2 / n3;
        const double a = cl * n1;
        const double n0 = fmin_f(a, n1);
        const double b = cl * n0;
        const double nm1 = fmin_f(b, n0);
        const double v1 = vs1[o + at(1)];
        const double rv0 = 2 * lo[s * ncol + c] - v1;
        const double rvm1 = rv0 + rv0 - v1;
        const double Tb0 = conv_re(n1, Ts[o + at(1)], s) / n1;
        const double gn0 = cn[at(0)], gnm1 = cn[at(-1)];
        const double grv0 = crv[at(0)], grvm1 = crv[at(-1)];
        const double gre0 = cre[at(0)], grem1 = cre[at(-1)];
        // re(0) = Tb0 n0, re(-1) = Tb0 nm1, Tb0 = re(1)/n(1)
        const double Tb0b = gre0 * n0 + grem1 * nm1;
        double N0 = gn0 + gre0 * Tb0, Nm1 = gnm1 + grem1 * Tb0;
        double g1 = -Tb0b * Tb0 / n1;  // -> n(1)
        cre[at(1)] += Tb0b / n1;
        // rv(0) = rv0 n0 ms, rv(-1) = rvm1 nm1 ms, rvm1 = 2 rv0 - v1, rv0 = 2 lo - v1
        double rv0b = grv0 * n0 * ms;
        N0 += grv0 * rv0 * ms;
        const double rvm1b = grvm1 * nm1 * ms;
        Nm1 += grvm1 * rvm1 * ms;
        rv0b += 2 * rvm1b;
        v1b1 += -rvm1b - rv0b;
        lob[s * ncol + c] = 2 * rv0b;
        // nm1 = min(cl n0, n0), n0 = min(cl n1, n1), cl = n2/n3
        double bb, n0b2;
        min_split(b, n0, Nm1, bb, n0b2);
        N0 += n0b2 + bb * cl;
        double clb = bb * n0;
        double ab, n1b2;
        min_split(a, n1, N0, ab, n1b2);
        g1 += n1b2 + ab * cl;
        clb += ab * n1;
        cn[at(1)] += g1;
        cn[at(2)] += clb / n3;
        cn[at(3)] += -clb * cl / n3;
        cn[at(0)] = cn[at(-1)] = 0.0;
        crv[at(0)] = crv[at(-1)] = 0.0;
        cre[at(0)] = cre[at(-1)] = 0.0;
      }
      // ---- top
      {
        const double nl = n[at(lx)], nl1 = n[at(lx - 1)], nl2 = n[at(lx - 2)];
        const double ch = nl1 / nl2;
        const double a = ch * nl;
        const double p1 = fmin_f(a, nl);
        const double b = ch * p1;
        const double p2 = fmin_f(b, p1);
        const double v1 = vs1[o + at(lx)];
        const double r1 = 2 * hi[s * ncol + c] - v1;
        const double r2 = r1 + r1 - v1;
        const double Tbl = conv_re(nl, Ts[o + at(lx)], s) / nl;
        const double gp1 = cn[at(lx + 1)], gp2 = cn[at(lx + 2)];
        const double gr1 = crv[at(lx + 1)], gr2 = crv[at(lx + 2)];
        const double ge1 = cre[at(lx + 1)], ge2 = cre[at(lx + 2)];
        const double Tblb = ge1 * p1 + ge2 * p2;
        double P1 = gp1 + ge1 * Tbl, P2 = gp2 + ge2 * Tbl;
        double gl = -Tblb * Tbl / nl;  // -> n(lx)
        cre[at(lx)] += Tblb / nl;
        double r1b = gr1 * p1 * ms;
        P1 += gr1 * r1 * ms;
        const double r2b = gr2 * p2 * ms;
        P2 += gr2 * r2 * ms;
        r1b += 2 * r2b;
        v1bl += -r2b - r1b;
        hib[s * ncol + c] = 2 * r1b;
        double bb, p1b2;
        min_split(b, p1, P2, bb, p1b2);
        P1 += p1b2 + bb * ch;
        double chb = bb * p1;
        double ab, nlb2;
        min_split(a, nl, P1, ab, nlb2);
        gl += nlb2 + ab * ch;
        chb += ab * nl;
        cn[at(lx)] += gl;
        cn[at(lx - 1)] += chb / nl2;
        cn[at(lx - 2)] += -chb * ch / nl2;
        cn[at(lx + 1)] = cn[at(lx + 2)] = 0.0;
        crv[at(lx + 1)] = crv[at(lx + 2)] = 0.0;
        cre[at(lx + 1)] = cre[at(lx + 2)] = 0.0;
      }
      vext[(2 * s) * ncol + c] = v1b1;
      vext[(2 * s + 1) * ncol + c] = v1bl;
    }
    if (Ttop_bar && s == 0) {
      double tsum = 0.0;
      for (int q = 0; q < LSP; ++q) tsum += ttb[q * ncol + c];
      Ttop_bar[c] = tsum;
    }
  }
}

// Adjoint of interface_vels for x1 (advec.f90:155-229) and of v12rhov1 / T2rhoe
// (multifluid.f90:193-214), writing the state cotangents (ghost cells 0), one thread per
// cell and species.  v1ib: the x1
// face cotangents of the three x1 sweep adjoints (n, rv, re slices of LSP*nf1 each, summed
// here); lob_out / hib_out: cotangents of the
// step's boundary-face outputs (may be null).
__global__ void ka_conv_vjp(GridDev G, const double* __restrict__ ns, const double* __restrict__ vs1,
                            const double* __restrict__ Ts, const double* __restrict__ C,
                            const double* __restrict__ v1ib, const double* __restrict__ lob_out,
                            const double* __restrict__ hib_out, const double* __restrict__ vext, double* nsb,
                            double* vs1b, double* Tsb) {
  const Dims d = G.d;
  const long long ng = d.ng;
  const long long ncol = (long long)d.lx2 * d.lx3;
  const long long nf = nf1(d);
  const int lx = d.lx1;
  for_rows_s(d, [&](long long k, int i1, int i2, int i3, bool in, int s) {
    const long long o = (long long)s * ng;
    if (!in) {
      nsb[o + k] = vs1b[o + k] = Tsb[o + k] = 0.0;
      return;
    }
    const long long col = (i2 - 1) + (long long)d.lx2 * (i3 - 1);
    {
      const double n = ns[o + k], v = vs1[o + k], T = Ts[o + k];
      const double gn = C[o + k], grv = C[LSP * ng + o + k], gre = C[2 * LSP * ng + o + k];
      const double ke = KB / (c_gammas[s] - 1);
      nsb[o + k] = gn + grv * c_ms[s] * v + gre * ke * T;
      Tsb[o + k] = gre * n * ke;
      // faces of this row: cotangent g(f), boundary outputs included
      auto gface = [&](int f) {
        const long long q = s * nf + f1i(d, f, i2, i3);
        double g = v1ib[q] + v1ib[LSP * nf + q] + v1ib[2 * LSP * nf + q];
        if (f == 1 && lob_out) g += lob_out[s * ncol + col];
        if (f == lx + 1 && hib_out) g += hib_out[s * ncol + col];
        return g;
      };
      double vb = grv * n * c_ms[s];
      if (i1 >= 2) vb += 0.5 * gface(i1);           // face i1 = (v(i1-1) + v(i1))/2
      if (i1 + 1 <= lx) vb += 0.5 * gface(i1 + 1);  // face i1+1 = (v(i1) + v(i1+1))/2
      const double* vr = vs1 + o;
      if (i1 <= 2) {  // face 1
        if (G.gridflag == 1) {
          const double mid = 0.5 * (vr[gi(d, 1, i2, i3)] + vr[gi(d, 2, i2, i3)]);
          const double w = (mid < 0.0) ? 1.0 : (mid == 0.0) ? 0.5 : 0.0;  // min(mid, 0)
          vb += 0.5 * w * gface(1);
        } else if (i1 == 1) {
          vb += gface(1);
        }
      }
      if (i1 >= lx - 1) {  // face lx+1
        if (G.gridflag == 2) {
          const double mid = 0.5 * (vr[gi(d, lx - 1, i2, i3)] + vr[gi(d, lx, i2, i3)]);
          const double w = (mid > 0.0) ? 1.0 : (mid == 0.0) ? 0.5 : 0.0;  // max(mid, 0)
          vb += 0.5 * w * gface(lx + 1);
        } else if (i1 == lx) {
          vb += gface(lx + 1);
        }
      }
      if (i1 == 1) vb += vext[(2 * s) * ncol + col];
      if (i1 == lx) vb += vext[(2 * s + 1) * ncol + col];
      vs1b[o + k] = vb;
    }
  });
}

}  // namespace gemk

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
struct gem_step_adjoint {
  const gem_grid* g = nullptr;
  long long F = 0;      // doubles of one 7-species ghosted field
  double* base = nullptr;
  double* WF = nullptr;  // fluidvars-shaped replay state (5F); reused by the backward
  double* ST = nullptr;  // four sweep stages, each n | rv | re (3F)
  double* CA = nullptr;  // cotangent stage (3F)
  double* CB = nullptr;  // its copy (3F)
  double *V1 = nullptr, *V2 = nullptr, *V3 = nullptr, *VP = nullptr, *VB = nullptr;  // faces
  double *vext = nullptr, *ttb = nullptr;
  // the three fields of a direction are swept concurrently: two side streams, fork/join events
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[2] = {nullptr, nullptr};
};

extern "C" {

int gem_step_adjoint_create(const gem_grid* g, gem_step_adjoint** out) {
  if (check_grid(g) || !out) return set_err(GEM_EINVAL, "null argument");
  *out = nullptr;
  int rc = check_step(g);
  if (rc) return rc;
  const Dims& d = g->dev.d;
  auto* a = new gem_step_adjoint();
  a->g = g;
  a->F = (long long)LSP * d.ng;
  const long long n1 = (long long)LSP * nf1(d), n2 = (long long)LSP * nf2(d), n3 = (long long)LSP * nf3(d);
  const long long ncol = (long long)d.lx2 * d.lx3;
  const long long total = 5 * a->F + 12 * a->F + 6 * a->F + 5 * n1 + n2 + n3 + 2 * LSP * ncol + LSP * ncol;
  if (cudaMalloc(&a->base, sizeof(double) * total) != cudaSuccess) {
    delete a;
    cudaGetLastError();
    return set_err(GEM_ENOMEM, "cudaMalloc of the step adjoint workspace (%lld doubles) failed", total);
  }
  double* p = a->base;
  a->WF = p;
  p += 5 * a->F;
  a->ST = p;
  p += 12 * a->F;
  a->CA = p;
  p += 3 * a->F;
  a->CB = p;
  p += 3 * a->F;
  a->V1 = p;
  p += n1;
  a->VP = p;
  p += n1;
  a->VB = p;  // three fields' vs1i cotangents
  p += 3 * n1;
  a->V2 = p;
  p += n2;
  a->V3 = p;
  p += n3;
  a->vext = p;
  p += 2 * LSP * ncol;
  a->ttb = p;
  // VP holds the stale boundary faces only; its other faces are never read, keep them finite
  GEM_CUDA(cudaMemset(a->VP, 0, sizeof(double) * n1));
  for (int i = 0; i < 2; ++i) {
    GEM_CUDA(cudaStreamCreateWithFlags(&a->side[i], cudaStreamNonBlocking));
    GEM_CUDA(cudaEventCreateWithFlags(&a->join[i], cudaEventDisableTiming));
  }
  GEM_CUDA(cudaEventCreateWithFlags(&a->fork, cudaEventDisableTiming));
  *out = a;
  return GEM_OK;
}

int gem_step_adjoint_destroy(gem_step_adjoint* a) {
  if (!a) return GEM_OK;
  for (int i = 0; i < 2; ++i) {
    if (a->side[i]) cudaStreamDestroy(a->side[i]);
    if (a->join[i]) cudaEventDestroy(a->join[i]);
  }
  if (a->fork) cudaEventDestroy(a->fork);
  cudaFree(a->base);
  delete a;
  return GEM_OK;
}

static int step_adjoint_check(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, const gem_step_adjoint* A) {
  if (!cfg || check_grid(g) || !w || !A) return set_err(GEM_EINVAL, "null argument");
  if (A->g != g) return set_err(GEM_EINVAL, "step adjoint workspace made for another grid");
  if (cfg->diffsolvetype != 1 && cfg->diffsolvetype != 2)
    return set_err(GEM_EINVAL, "Unsupported diffusion solver type/mode: %d. Should be either 1 or 2.", cfg->diffsolvetype);
  if (g->dev.has_null) return set_err(GEM_EINVAL, "the step adjoint supports grids without null cells");
  return check_step(g);
}

int gem_step_vjp_replay_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* A,
                            const double* ns, const double* vs1, const double* vs2, const double* vs3,
                            const double* Ts, const double* v1i_lo, const double* v1i_hi, const double* dt,
                            void* stream) {
  int rc0 = step_adjoint_check(cfg, g, w, A);
  if (rc0) return rc0;
  if (!ns || !vs1 || !vs2 || !vs3 || !Ts || !v1i_lo || !v1i_hi || !dt) return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  const GridDev& G = g->dev;
  const Dims& d = G.d;
  const long long F = A->F;
  const unsigned ngb = grid_for(d.ng, 256);
  const long long ncol = (long long)d.lx2 * d.lx3;
  double* WF = A->WF;
  double* Sx[4] = {A->ST, A->ST + 3 * F, A->ST + 6 * F, A->ST + 9 * F};
  const int dims[3] = {3, 1, 2};
  const double* vel[3] = {A->V3, A->V1, A->V2};
  int rc = GEM_OK;
  const size_t FB = sizeof(double) * F;
  double* S0 = A->ST;
  // ---------------- forward replay
  GEM_CUDA(cudaMemcpyAsync(WF, ns, FB, cudaMemcpyDeviceToDevice, st));
  GEM_CUDA(cudaMemcpyAsync(WF + F, vs1, FB, cudaMemcpyDeviceToDevice, st));
  GEM_CUDA(cudaMemcpyAsync(WF + 2 * F, vs2, FB, cudaMemcpyDeviceToDevice, st));
  GEM_CUDA(cudaMemcpyAsync(WF + 3 * F, vs3, FB, cudaMemcpyDeviceToDevice, st));
  GEM_CUDA(cudaMemcpyAsync(WF + 4 * F, Ts, FB, cudaMemcpyDeviceToDevice, st));
  ka_set_faces<<<grid_for(ncol * LSP, 256), 256, 0, st>>>(d, v1i_lo, v1i_hi, A->VP);
  GEM_LAUNCHED("ka_set_faces");
  Blocks B = blocks(g, WF, S0 + F);  // rv, re straight into stage 0
  k_v12rhov1<<<ngb, 256, 0, st>>>(B);
  GEM_LAUNCHED("k_v12rhov1");
  k_T2rhoe<<<ngb, 256, 0, st>>>(B);
  GEM_LAUNCHED("k_T2rhoe");
  if ((rc = launch_ghost_fill(g, B, A->VP, LSP, false, st))) return rc;
  if (G.flagper) {
    k_halo_wrap<<<grid_for((long long)(d.lx1 + 4) * d.lx2 * LSP, 256), 256, 0, st>>>(G, B, 1);
    GEM_LAUNCHED("k_halo_wrap");
  }
  GEM_CUDA(cudaMemcpyAsync(S0, WF, FB, cudaMemcpyDeviceToDevice, st));
  k_interface_vels<<<dim3(grid_for(nf1(d) + nf2(d) + nf3(d), 256, 4), LSP), 256, 0, st>>>(G, B, A->V1, A->V2,
                                                                                         A->V3);
  GEM_LAUNCHED("k_interface_vels");
  // the nine sweeps: (dim, velocities) per stage, fields n (frank 0, 6 species), rv (frank 1
  // for x2/x3, 6 species), re (frank 0, 7 species)
  for (int q = 0; q < 3; ++q) {
    double* Sin = Sx[q];
    double* So = Sx[q + 1];
    // fork: field 0 on the caller's stream, fields 1 and 2 on the side streams
    GEM_CUDA(cudaEventRecord(A->fork, st));
    for (int i = 0; i < 2; ++i) GEM_CUDA(cudaStreamWaitEvent(A->side[i], A->fork, 0));
    for (int fld = 0; fld < 3; ++fld) {
      cudaStream_t fs = (fld == 0) ? st : A->side[fld - 1];
      GEM_CUDA(cudaMemcpyAsync(So + fld * F, Sin + fld * F, FB, cudaMemcpyDeviceToDevice, fs));
      const int frank = (fld == 1 && dims[q] != 1) ? 1 : 0;
      SweepArgs sa;
      Blocks fb;
      fb.F = fb.A = So + fld * F;
      fb.ng = d.ng;
      sa.G = G;
      sa.B = fb;
      sa.vsi = vel[q];
      sa.vs1i = nullptr;
      sa.dtp = dt;
      sa.dtp_w = nullptr;
      sa.which = frank;
      if ((rc = launch_sweep(g, dims[q], false, sa, fld == 2 ? LSP : LSP - 1, fs))) return rc;
    }
    for (int i = 0; i < 2; ++i) {  // join
      GEM_CUDA(cudaEventRecord(A->join[i], A->side[i]));
      GEM_CUDA(cudaStreamWaitEvent(st, A->join[i], 0));
    }
    if (q == 1 && G.flagper) {  // halo_allparams self-wrap between the x1 and x2 sweeps
      Blocks wb = blocks(g, So, So + F);
      k_halo_wrap<<<grid_for((long long)(d.lx1 + 4) * d.lx2 * LSP, 256), 256, 0, st>>>(G, wb, 0);
      GEM_LAUNCHED("k_halo_wrap");
    }
  }
  // the post-sweep values the diffusion adjoint needs (WF's state copy is dead now)
  double* NO = WF;
  double* TP = WF + F;
  ka_post_fwd<<<ngb, 256, 0, st>>>(G, Sx[3], NO, TP);
  GEM_LAUNCHED("ka_post_fwd");
  return GEM_OK;
}

int gem_step_vjp_finish_dev(const gem_cfg* cfg, const gem_grid* g, gem_work* w, const gem_step_adjoint* A,
                            double* fluidvars, double* fluidauxvars, const double* electrovars, const double* dt,
                            double* v1i_lo, double* v1i_hi, void* stream) {
  int rc = step_adjoint_check(cfg, g, w, A);
  if (rc) return rc;
  if (!fluidvars || !fluidauxvars || !electrovars || !dt || !v1i_lo || !v1i_hi)
    return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  const GridDev& G = g->dev;
  const Dims& d = G.d;
  const long long ncol = (long long)d.lx2 * d.lx3;
  Blocks B = blocks(g, fluidvars, fluidauxvars);
  // the x2 sweep's epilogue from the replay's last stage, then the rest of gem_fluid_adv_dev
  ka_finish_fwd<<<grid_for(d.ng, 256), 256, 0, st>>>(G, A->ST + 9 * A->F, B);
  GEM_LAUNCHED("ka_finish_fwd");
  k_ghost_epilogue<<<grid_for(ghost_cells(d), 256), 256, 0, st>>>(G, B);
  GEM_LAUNCHED("k_ghost_epilogue");
  if (G.has_null && (G.gridflag == 0 || G.gridflag == 1)) {
    k_clean_vel_edges<<<grid_for(ncol * LSP, 128), 128, 0, st>>>(G, fluidvars + LSP * d.ng);
    GEM_LAUNCHED("k_clean_vel_edges");
  }
  DiffArgs da;
  da.G = G;
  da.B = B;
  da.J1 = electrovars + 3 * d.ng;
  da.nn = w->nn;
  da.Tn = w->Tn;
  da.dtp = dt;
  da.Teinf = cfg->Teinf;
  da.Ttop = w->Ttop;
  if ((rc = work_lu(w, g, &da.lu))) return rc;
  da.solver = cfg->diffsolvetype;
  da.fused = 1;
  if ((rc = launch_diffusion(g, da, st))) return rc;
  // the boundary faces the forward's x1 sweep stores for the next step: the replay's x1
  // interface velocities there (the same formulas, advec.f90:170-196)
  ka_get_faces<<<grid_for(ncol * LSP, 256), 256, 0, st>>>(d, A->V1, v1i_lo, v1i_hi);
  GEM_LAUNCHED("ka_get_faces");
  return GEM_OK;
}

int gem_step_vjp_backward_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* A,
                              const double* ns, const double* vs1, const double* Ts, const double* v1i_lo,
                              const double* v1i_hi, const double* electrovars, const double* dt,
                              const double* ns_bar_out, const double* vs1_bar_out, const double* Ts_bar_out,
                              const double* lo_bar_out, const double* hi_bar_out, double* ns_bar, double* vs1_bar,
                              double* Ts_bar, double* lo_bar, double* hi_bar, double* Ttop_bar, void* stream) {
  int rc0 = step_adjoint_check(cfg, g, w, A);
  if (rc0) return rc0;
  if (!ns || !vs1 || !Ts || !v1i_lo || !v1i_hi || !electrovars || !dt || !ns_bar_out || !vs1_bar_out ||
      !Ts_bar_out || !ns_bar || !vs1_bar || !Ts_bar || !lo_bar || !hi_bar)
    return set_err(GEM_EINVAL, "null argument");
  cudaStream_t st = S(stream);
  const GridDev& G = g->dev;
  const Dims& d = G.d;
  const long long F = A->F;
  const unsigned ngb = grid_for(d.ng, 256);
  const long long ncol = (long long)d.lx2 * d.lx3;
  double* WF = A->WF;
  double* Sx[4] = {A->ST, A->ST + 3 * F, A->ST + 6 * F, A->ST + 9 * F};
  const int dims[3] = {3, 1, 2};
  const double* vel[3] = {A->V3, A->V1, A->V2};
  int rc = GEM_OK;
  // ---------------- backward
  double* NO = WF;           // n after clean_param(1) (from the replay)
  double* TP = WF + F;       // T into the diffusion (from the replay)
  double* TPB = WF + 2 * F;  // its cotangent
  double* NDB = WF + 3 * F;  // cotangent of the diffusion's n input
  {
    DiffAdjArgs da;
    da.G = G;
    da.T = TP;
    da.ns = NO;
    da.J1 = electrovars + 3 * d.ng;
    da.nn = w->nn;
    da.Tn = w->Tn;
    da.Ttop = w->Ttop;
    da.Teinf = cfg->Teinf;
    da.dtp = dt;
    da.solver = cfg->diffsolvetype;
    da.Ybar = Ts_bar_out;
    da.Tbar = TPB;
    da.nbar = NDB;
    da.Ttop_bar = Ttop_bar ? A->ttb : nullptr;
    if ((rc = launch_diffusion_vjp(g, da, st))) return rc;
  }
  double* C = A->CA;
  double* Cn = A->CB;
  ka_post_vjp<<<ngb, 256, 0, st>>>(G, Sx[3], ns_bar_out, vs1_bar_out, TPB, NDB, C);
  GEM_LAUNCHED("ka_post_vjp");
  const long long nvf = (long long)LSP * nf1(d);  // one field's vs1i cotangent slice
  GEM_CUDA(cudaMemsetAsync(A->VB, 0, sizeof(double) * 3 * nvf, st));
  for (int q = 2; q >= 0; --q) {
    if (q == 1 && G.flagper) {
      ka_wrap3_vjp<<<grid_for((long long)(d.lx1 + 4) * d.lx2 * 3 * LSP, 256), 256, 0, st>>>(G, C);
      GEM_LAUNCHED("ka_wrap3_vjp");
    }
    if (dims[q] == 1)
      ka_frame_copy<1><<<ngb, 256, 0, st>>>(G, C, Cn);
    else if (dims[q] == 2)
      ka_frame_copy<2><<<ngb, 256, 0, st>>>(G, C, Cn);
    else
      ka_frame_copy<3><<<ngb, 256, 0, st>>>(G, C, Cn);
    GEM_LAUNCHED("ka_frame_copy");
    // the three fields in one launch; x1 also gives each field's vs1i cotangent (its own
    // slice of VB, summed by ka_conv_vjp); the x2/x3 velocities are fixed
    SweepVjpFields FS;
    for (int fld = 0; fld < 3; ++fld) {
      FS.f[fld] = Sx[q] + fld * F;
      FS.obar[fld] = C + fld * F;
      FS.fbar[fld] = Cn + fld * F;
      FS.vbar[fld] = (dims[q] == 1) ? A->VB + fld * nvf : nullptr;
      FS.nsp[fld] = fld == 2 ? LSP : LSP - 1;
      FS.frank[fld] = (fld == 1 && dims[q] != 1) ? 1 : 0;
    }
    FS.nfld = 3;
    FS.nfs = 3 * LSP - 2;
    if (dims[q] == 1) {
      if ((rc = launch_sweep_vjp_x1(g, FS, vel[q], dt, 0, st))) return rc;
    } else {
      if ((rc = launch_sweep_vjp_march(g, dims[q], FS, vel[q], dt, nullptr, 0, st))) return rc;
    }
    std::swap(C, Cn);
  }
  // the ghost fill's x3 pass: edge copies, or the periodic self-wrap
  if (G.flagper) {
    ka_wrap3_vjp<<<grid_for((long long)(d.lx1 + 4) * d.lx2 * 3 * LSP, 256), 256, 0, st>>>(G, C);
    GEM_LAUNCHED("ka_wrap3_vjp");
  } else {
    ka_copy_vjp<3><<<grid_for((long long)(d.lx1 + 4) * (d.lx2 + 4) * 3 * LSP, 256), 256, 0, st>>>(G, C);
    GEM_LAUNCHED("ka_copy_vjp<3>");
  }
  ka_copy_vjp<2><<<grid_for((long long)(d.lx1 + 4) * (d.lx3 + 4) * 3 * LSP, 256), 256, 0, st>>>(G, C);
  GEM_LAUNCHED("ka_copy_vjp<2>");
  ka_x1bc_vjp<<<grid_for(ncol * LSP, 128), 128, 0, st>>>(G, ns, vs1, Ts, v1i_lo, v1i_hi, C, A->vext, lo_bar, hi_bar,
                                                    Ttop_bar ? A->ttb : nullptr, Ttop_bar);
  GEM_LAUNCHED("ka_x1bc_vjp");
  ka_conv_vjp<<<ngb, 256, 0, st>>>(G, ns, vs1, Ts, C, A->VB, lo_bar_out, hi_bar_out, A->vext, ns_bar, vs1_bar,
                                   Ts_bar);
  GEM_LAUNCHED("ka_conv_vjp");
  return GEM_OK;
}

int gem_step_vjp_dev(const gem_cfg* cfg, const gem_grid* g, const gem_work* w, gem_step_adjoint* A,
                     const double* ns, const double* vs1, const double* vs2, const double* vs3, const double* Ts,
                     const double* v1i_lo, const double* v1i_hi, const double* electrovars, const double* dt,
                     const double* ns_bar_out, const double* vs1_bar_out, const double* Ts_bar_out,
                     const double* lo_bar_out, const double* hi_bar_out, double* ns_bar, double* vs1_bar,
                     double* Ts_bar, double* lo_bar, double* hi_bar, double* Ttop_bar, void* stream) {
  int rc = gem_step_vjp_replay_dev(cfg, g, w, A, ns, vs1, vs2, vs3, Ts, v1i_lo, v1i_hi, dt, stream);
  if (rc) return rc;
  return gem_step_vjp_backward_dev(cfg, g, w, A, ns, vs1, Ts, v1i_lo, v1i_hi, electrovars, dt, ns_bar_out,
                                   vs1_bar_out, Ts_bar_out, lo_bar_out, hi_bar_out, ns_bar, vs1_bar, Ts_bar, lo_bar,
                                   hi_bar, Ttop_bar, stream);
}

}  // extern "C"
