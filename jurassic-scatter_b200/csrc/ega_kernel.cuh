// The EGA + continua + Planck + radiative-transfer kernel: a thread per
// (ray, channel), serial along the ray because the EGA carries the path
// transmittance (src/forwardmodel.c:302-399, :409-565; continua
// src/forwardmodel.c:120-152; Planck source :743-794).  Each emitter-count
// instantiation lives in its own translation unit (ega_g*.cu) so they
// compile in parallel.
#pragma once
#include "device_common.cuh"

// One thread per (ray, channel).  The path state of every emitter lives in
// registers (GMAX >= ng, the emitter loop is unrolled so the lookups of
// different emitters overlap); LOS records are read by all threads of a
// ray (broadcast loads).
template <int GMAX, bool DIG, int BLK, int MINB, bool ROLL>
__global__ void __launch_bounds__(BLK, MINB) ega_rt_kernel(EgaArgs A) {
  const jsc_dev_model &m = A.m;
  const int nd = m.nd, ng = m.ng;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = tid / A.ndp;
  const int d = tid - r * A.ndp;
  if (r >= A.n_rays || d >= nd) return;

  // per-channel constants
  const int w = m.window[d];
  const bool has_w = w < m.nw;
  const jsc_ctm_coef cc = m.ctm[d];
  const double nu = m.nu[d];
  const double *__restrict__ pb = m.planck_b + (size_t)d * JSC_NPLANCK;
  const double *__restrict__ ps = m.planck_s + (size_t)d * JSC_NPLANCK;
  const jsc_row *__restrict__ rows_d = m.rows + d;  // [ip][it][g][d]
  const size_t rs = (size_t)ng * nd;                 // stride of one (ip, it) slot
  unsigned okmask = 0;
  for (int g = 0; g < ng && g < GMAX; g++)
    if (m.tab_grid[d * ng + g] >= 0) okmask |= 1u << g;

  // Path transmittance and interval hints per emitter: registers
  // (unrolled) or local memory (rolled).  (State in shared memory measured
  // slower: the allocation shrinks the L1 the table gathers hit.)
  double tp_l[GMAX];
  // four 16-bit interval hints per emitter, one per (p, T) corner row:
  // rows one pressure level apart sit several intervals apart on the
  // column-density grid, so a shared hint sends three of them searching
  unsigned long long hint_l[GMAX];
  // per emitter: the (p, T) bracket code the hints belong to, and the
  // forward distances j - k of the four rows (8 bits each)
  int hcode_l[GMAX];
  unsigned dj_l[GMAX];
#define JSC_TP(g) (tp_l[g])
#define JSC_HINT(g) (hint_l[g])
#pragma unroll((GMAX <= 8 && !ROLL) ? GMAX : 1)
  for (int g = 0; g < GMAX; g++) {
    JSC_TP(g) = 1;
    JSC_HINT(g) = 0;
    hcode_l[g] = -1;
    dj_l[g] = 0;
  }
  double rad = 0, tau = 1;
  unsigned long long dig[DIG ? GMAX : 1];  // per-emitter index digests
#pragma unroll
  for (int g = 0; g < (DIG ? GMAX : 1); g++) dig[g] = 0;
  unsigned n_ega = 0;
  const int np = A.nlos[r];
  const double *__restrict__ rec = A.pts + (size_t)A.los_off[r] * A.W;
  // scattering source of this ray's next scattering point
  const double *__restrict__ ssrc = A.src_sca ? A.src_sca + (size_t)A.sp_off[r] * nd + d : nullptr;

  for (int ip = 0; ip < np; ip++, rec += A.W) {
    const double P = rec[REC_P], T = rec[REC_T], DS = rec[REC_DS];
    const int itp = (int)rec[REC_PLK];
    int code = (int)rec[REC_GRID];
    double tau_gas = 1;
    // unrolled up to 8 emitters (state in registers, lookups of different
    // emitters overlap) unless ROLL; larger counts and ROLL keep the state in
    // local memory and the code small
#pragma unroll((GMAX <= 8 && !ROLL) ? GMAX : 1)
    for (int g = 0; g < GMAX; g++) {
      if (g >= ng) break;
      double eps = 0;
      const double tpg = JSC_TP(g);
      if (!((okmask >> g) & 1u)) {
        eps = 0;
      } else if (tpg < 1e-9) {
        eps = 1;
      } else {
        const int gid = A.single_grid ? 0 : m.tab_grid[d * ng + g];
        if (!A.single_grid)
          code = grid_code(m.grid_np[gid], m.grid_p + (size_t)gid * TBLNPMAX,
                           m.grid_nt + (size_t)gid * TBLNPMAX,
                           m.grid_t + (size_t)gid * TBLNPMAX * TBLNTMAX, P, T);
        if (code & (1 << 16)) {
          const int ipr = (code >> 10) & 63, it0 = (code >> 5) & 31, it1 = code & 31;
          const jsc_row *rw = rows_d + (size_t)g * nd;
          const jsc_row r00 = rw[(size_t)(ipr * TBLNTMAX + it0) * rs];
          const jsc_row r01 = rw[(size_t)(ipr * TBLNTMAX + it0 + 1) * rs];
          const jsc_row r10 = rw[(size_t)((ipr + 1) * TBLNTMAX + it1) * rs];
          const jsc_row r11 = rw[(size_t)((ipr + 1) * TBLNTMAX + it1 + 1) * rs];
          if ((r00.nf & 0xffff) >= 2 && (r01.nf & 0xffff) >= 2 &&
              (r10.nf & 0xffff) >= 2 && (r11.nf & 0xffff) >= 2) {
            const double x1 = 1 - tpg, useg = rec[REC_K + m.nw + g];
            unsigned long long *dg = &dig[DIG ? g : 0];
            if (DIG) *dg = *dg * 1000003ull + (unsigned long long)(ipr * 961 + it0 * 31 + it1);
            unsigned long long hp = JSC_HINT(g);
            const int hc = hcode_l[g];
            if (hc >= 0 && hc != code) hp = remap_hints(hp, hc, code);
            const unsigned dj = dj_l[g];
            int k00, k01, k10, k11, j00, j01, j10, j11;
            const double e00 = ega_node<DIG, ROLL>(m.nodes, r00, x1, useg, (int)(hp & 0xffff),
                                             (int)(dj & 0xff), &k00, &j00, dg);
            const double e01 = ega_node<DIG, ROLL>(m.nodes, r01, x1, useg, (int)((hp >> 16) & 0xffff),
                                             (int)((dj >> 8) & 0xff), &k01, &j01, dg);
            const double e10 = ega_node<DIG, ROLL>(m.nodes, r10, x1, useg, (int)((hp >> 32) & 0xffff),
                                             (int)((dj >> 16) & 0xff), &k10, &j10, dg);
            const double e11 = ega_node<DIG, ROLL>(m.nodes, r11, x1, useg, (int)(hp >> 48),
                                             (int)(dj >> 24), &k11, &j11, dg);
            JSC_HINT(g) = (unsigned long long)(j00 & 0xffff) | ((unsigned long long)(j01 & 0xffff) << 16) |
                          ((unsigned long long)(j10 & 0xffff) << 32) |
                          ((unsigned long long)(j11 & 0xffff) << 48);
            hcode_l[g] = code;
            dj_l[g] = (unsigned)min(j00 - k00, 255) | ((unsigned)min(j01 - k01, 255) << 8) |
                      ((unsigned)min(j10 - k10, 255) << 16) | ((unsigned)min(j11 - k11, 255) << 24);
            const double *gp = m.grid_p + (size_t)gid * TBLNPMAX;
            const double *gt = m.grid_t + (size_t)gid * TBLNPMAX * TBLNTMAX;
            double ea = jsc_clamp01(jsc_lin(gt[ipr * TBLNTMAX + it0], e00,
                                            gt[ipr * TBLNTMAX + it0 + 1], e01, T));
            const double eb = jsc_clamp01(jsc_lin(gt[(ipr + 1) * TBLNTMAX + it1], e10,
                                                  gt[(ipr + 1) * TBLNTMAX + it1 + 1], e11, T));
            ea = jsc_clamp01(jsc_lin(gp[ipr], ea, gp[ipr + 1], eb, P));
            eps = 1 - (1 - ea) / tpg;
            n_ega++;
          }
        }
      }
      JSC_TP(g) = tpg * (1 - eps);
      tau_gas *= (1 - eps);
    }
    const double beta = continua(m, A.cfg, cc, nu, has_w ? rec[REC_K + w] : 0.0, P, T, DS,
                                 rec[REC_QH2O], rec + REC_K + m.nw);
    const double src = pb[itp] + ps[itp] * (T - planck_temp(itp));
    const double af = rec[REC_AF];
    if (ssrc && af > 0) {
      // scattering point: gas, continuum and aerosol extinction, thermal
      // source mixed with the scattering source by the single-scattering
      // albedo of the layer (src/forwardmodel.c:317-363)
      if (tau_gas > 0) {
        const int ia = (int)rec[REC_AI];
        const double be = A.beta[ia * nd + d], bs = A.beta[A.aero_nl * nd + ia * nd + d];
        const double bext = (-1.) * log(tau_gas) / DS + beta + af * be;
        const double eps = 1 - exp(-1 * bext * DS);
        const double src_all = ((bext - af * bs) * src + af * bs * *ssrc) / bext;
        rad += tau * eps * src_all;
        tau *= exp(-1. * bext * DS);
      }
      ssrc += nd;
    } else if (tau_gas > 0) {
      // clear air, or aerosol/cloud extinction without a scattering source
      // (src/forwardmodel.c:365-389)
      double eps;
      if (A.cfg.sca_n == 0 || af == 0) {
        eps = 1 - tau_gas * exp(-1. * beta * DS);
      } else {
        const int ia = (int)rec[REC_AI];
        const double bx = A.beta[(A.cfg.sca_ext_beta_a ? 2 : 0) * A.aero_nl * nd + ia * nd + d];
        eps = 1 - tau_gas * exp(-1. * (beta + af * bx) * DS);
      }
      rad += src * eps * tau;
      tau *= (1 - eps);
    }
  }
#undef JSC_TP
#undef JSC_HINT
  const double ts = A.tsurf[r];
  if (ts > 0) {
    const int its = planck_index(ts);
    rad += (pb[its] + ps[its] * (ts - planck_temp(its))) * tau;
  }
  A.rad[(size_t)r * nd + d] = rad;
  A.tau[(size_t)r * nd + d] = tau;
  if (DIG) {
    // fold of the per-emitter digests in emitter order
    unsigned long long dd = 0;
    for (int g = 0; g < ng && g < GMAX; g++) dd = dd * 1000003ull + dig[g];
    A.digest[(size_t)r * nd + d] = dd;
  }
  const unsigned mask = __activemask();
  const unsigned tot = __reduce_add_sync(mask, n_ega);
  if ((threadIdx.x & 31) == __ffs(mask) - 1) atomicAdd(&A.counters[1], (unsigned long long)tot);
}

// Launch variants: (threads per block, minimum resident blocks per SM);
// the second number sets the register budget, i.e. the trade between
// occupancy and spills.  jsc_batch_autotune picks one.
template <int G, bool DIG>
static void ega_launch_variant(const EgaArgs &ea, unsigned g128, unsigned g256, int v,
                               cudaStream_t s) {
  switch (v) {
    case 0: ega_rt_kernel<G, DIG, 128, 4, false><<<g128, 128, 0, s>>>(ea); break;
    case 2: ega_rt_kernel<G, DIG, 128, 8, false><<<g128, 128, 0, s>>>(ea); break;
    case 3: ega_rt_kernel<G, DIG, 256, 3, false><<<g256, 256, 0, s>>>(ea); break;
    case 4: ega_rt_kernel<G, DIG, 256, 4, false><<<g256, 256, 0, s>>>(ea); break;
    case 5: ega_rt_kernel<G, DIG, 128, 8, true><<<g128, 128, 0, s>>>(ea); break;
    case 6: ega_rt_kernel<G, DIG, 128, 12, true><<<g128, 128, 0, s>>>(ea); break;
    case 7: ega_rt_kernel<G, DIG, 256, 4, true><<<g256, 256, 0, s>>>(ea); break;
    case 8: ega_rt_kernel<G, DIG, 256, 6, true><<<g256, 256, 0, s>>>(ea); break;
    default: ega_rt_kernel<G, DIG, 128, 6, false><<<g128, 128, 0, s>>>(ea); break;
  }
}

// Launchers, one per emitter-count bound (defined in ega_g*.cu).
void jsc_ega_launch_g2(const EgaArgs &, unsigned, unsigned, int, bool, cudaStream_t);
void jsc_ega_launch_g4(const EgaArgs &, unsigned, unsigned, int, bool, cudaStream_t);
void jsc_ega_launch_g8(const EgaArgs &, unsigned, unsigned, int, bool, cudaStream_t);
void jsc_ega_launch_gmax(const EgaArgs &, unsigned, unsigned, int, bool, cudaStream_t);

// Default variant of this kernel family: 128 threads, 12 blocks per SM,
// rolled emitter loop.  Index digests run the selected variant (every
// variant has a digest instance).
#define JSC_EGA_DEFAULT_VARIANT 6
#define JSC_EGA_LAUNCHER(NAME, G)                                                      \
  void NAME(const EgaArgs &ea, unsigned g128, unsigned g256, int v, bool dig,          \
            cudaStream_t s) {                                                          \
    if (dig) ega_launch_variant<G, true>(ea, g128, g256, v, s);                        \
    else ega_launch_variant<G, false>(ea, g128, g256, v, s);                           \
  }
