// The EGA + radiative-transfer kernel with lanes over (channel, emitter),
// and the per-(LOS point, channel) continuum and Planck kernel it reads.
//
// ctm_src_kernel   one thread per (LOS point, channel): continuum extinction
//                  (src/forwardmodel.c:120-152) and Planck source
//                  (:788-793), written [point][channel].
// ega_lane_kernel  a group of GP lanes per (ray, channel), one lane per
//                  emitter: each lane carries its emitter's path
//                  transmittance along the ray and evaluates its EGA
//                  (src/forwardmodel.c:409-502); the group multiplies the
//                  segment transmittances in emitter order (shuffles) and
//                  every lane of the group runs the same radiative transfer
//                  step (:302-399); lane 0 writes the result.
//
// One emitter per lane keeps the path state in registers (no local
// arrays), the loop body small and the number of independent table
// gathers in flight per SM high; the continua, whose transcendental
// functions cost more than the EGA itself, run once per (point, channel)
// in a separate, fully parallel launch.
#pragma once
#include "device_common.cuh"

struct CtmArgs {
  jsc_dev_model m;
  jsc_run_cfg cfg;
  int64_t n_points;
  int W;
  const double *pts;
  double *beta, *src;  // [n_points][nd]
  const int64_t *n_live;  // LOS points on the device (fixed-capacity runs), or null
};

static __global__ void __launch_bounds__(256) ctm_src_kernel(CtmArgs A) {
  const int nd = A.m.nd;
  const int64_t total = (A.n_live ? *A.n_live : A.n_points) * nd;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t pt = t / nd;
    const int d = (int)(t - pt * nd);
    const double *rec = A.pts + pt * A.W;
    const double P = rec[REC_P], T = rec[REC_T], DS = rec[REC_DS];
    const int w = A.m.window[d];
    A.beta[t] = continua(A.m, A.cfg, A.m.ctm[d], A.m.nu[d], w < A.m.nw ? rec[REC_K + w] : 0.0, P,
                         T, DS, rec[REC_QH2O], rec + REC_K + A.m.nw);
    const int itp = (int)rec[REC_PLK];
    A.src[t] = planck_src(A.m, d, itp, T);
  }
}

// Path state of one (ray, channel, emitter) along its ray: the emitter's
// path transmittance, a 16-bit interval hint per (p, T) corner row and the
// bracket code the hints belong to, the forward distances j - k of the
// rows (8 bits each), the index digest and the EGA evaluation count.
struct EgaPath {
  double tp;
  unsigned long long hint;
  int hcode;
  unsigned djp;
  unsigned long long dig;
  unsigned n_ega;
};

__device__ __forceinline__ EgaPath ega_path_start() {
  EgaPath ps;
  ps.tp = 1;
  ps.hint = 0;
  ps.hcode = -1;
  ps.djp = 0;
  ps.dig = 0;
  ps.n_ega = 0;
  return ps;
}

// The emissivity table of (channel d, emitter g): its grid id (ok: the
// table exists), its (ip, it) row descriptors with the stride of one slot,
// and its pressure and temperature grids.
struct EgaTable {
  int gid;
  bool ok;
  const jsc_row *__restrict__ rows_dg;
  size_t rs;
  const double *__restrict__ gp;
  const double *__restrict__ gt;
};

__device__ __forceinline__ EgaTable ega_table(const jsc_dev_model &m, int d, int g) {
  EgaTable tb;
  const bool has_g = g < m.ng;
  tb.gid = has_g ? m.tab_grid[d * m.ng + g] : -1;
  tb.ok = tb.gid >= 0;
  tb.rows_dg = m.rows + (size_t)(has_g ? g : 0) * m.nd + d;
  tb.rs = (size_t)m.ng * m.nd;
  tb.gp = m.grid_p + (size_t)(tb.ok ? tb.gid : 0) * TBLNPMAX;
  tb.gt = m.grid_t + (size_t)(tb.ok ? tb.gid : 0) * TBLNPMAX * TBLNTMAX;
  return tb;
}

// Segment emissivity of one emitter at the LOS point rec (intpol_tbl,
// src/forwardmodel.c:409-502): the four (p, T) corner rows, each an
// inverse lookup of the path emissivity and a forward lookup of the
// extended column (ega_node), interpolated in T, then in p; the path
// state's hints and digest advance.  The caller multiplies ps.tp by
// (1 - eps).
template <bool DIG>
__device__ __forceinline__ double ega_lane_eps(const jsc_dev_model &m, bool single_grid,
                                               const EgaTable &tb, int g,
                                               const double *__restrict__ rec, EgaPath &ps) {
  const double P = rec[REC_P], T = rec[REC_T];
  double eps = 0;
  if (tb.ok) {
    if (ps.tp < 1e-9) {
      eps = 1;
    } else {
      const int code = single_grid
                           ? (int)rec[REC_GRID]
                           : grid_code(m.grid_np[tb.gid], tb.gp,
                                       m.grid_nt + (size_t)tb.gid * TBLNPMAX, tb.gt, P, T);
      if (code & (1 << 16)) {
        const int ipr = (code >> 10) & 63, it0 = (code >> 5) & 31, it1 = code & 31;
        const jsc_row r00 = tb.rows_dg[(size_t)(ipr * TBLNTMAX + it0) * tb.rs];
        const jsc_row r01 = tb.rows_dg[(size_t)(ipr * TBLNTMAX + it0 + 1) * tb.rs];
        const jsc_row r10 = tb.rows_dg[(size_t)((ipr + 1) * TBLNTMAX + it1) * tb.rs];
        const jsc_row r11 = tb.rows_dg[(size_t)((ipr + 1) * TBLNTMAX + it1 + 1) * tb.rs];
        if ((r00.nf & 0xffff) >= 2 && (r01.nf & 0xffff) >= 2 && (r10.nf & 0xffff) >= 2 &&
            (r11.nf & 0xffff) >= 2) {
          const double x1 = 1 - ps.tp, useg = rec[REC_K + m.nw + g];
          if (DIG) ps.dig = ps.dig * 1000003ull + (unsigned long long)(ipr * 961 + it0 * 31 + it1);
          if (ps.hcode >= 0 && ps.hcode != code) ps.hint = remap_hints(ps.hint, ps.hcode, code);
          int k00, k01, k10, k11, j00, j01, j10, j11;
          const double e00 = ega_node<DIG>(m.nodes, r00, x1, useg, (int)(ps.hint & 0xffff),
                                           (int)(ps.djp & 0xff), &k00, &j00, &ps.dig);
          const double e01 = ega_node<DIG>(m.nodes, r01, x1, useg, (int)((ps.hint >> 16) & 0xffff),
                                           (int)((ps.djp >> 8) & 0xff), &k01, &j01, &ps.dig);
          const double e10 = ega_node<DIG>(m.nodes, r10, x1, useg, (int)((ps.hint >> 32) & 0xffff),
                                           (int)((ps.djp >> 16) & 0xff), &k10, &j10, &ps.dig);
          const double e11 = ega_node<DIG>(m.nodes, r11, x1, useg, (int)(ps.hint >> 48),
                                           (int)(ps.djp >> 24), &k11, &j11, &ps.dig);
          ps.hint = (unsigned long long)(j00 & 0xffff) |
                    ((unsigned long long)(j01 & 0xffff) << 16) |
                    ((unsigned long long)(j10 & 0xffff) << 32) |
                    ((unsigned long long)(j11 & 0xffff) << 48);
          ps.hcode = code;
          ps.djp = (unsigned)min(j00 - k00, 255) | ((unsigned)min(j01 - k01, 255) << 8) |
                   ((unsigned)min(j10 - k10, 255) << 16) | ((unsigned)min(j11 - k11, 255) << 24);
          double ea = jsc_clamp01(jsc_lin(tb.gt[ipr * TBLNTMAX + it0], e00,
                                          tb.gt[ipr * TBLNTMAX + it0 + 1], e01, T));
          const double eb = jsc_clamp01(jsc_lin(tb.gt[(ipr + 1) * TBLNTMAX + it1], e10,
                                                tb.gt[(ipr + 1) * TBLNTMAX + it1 + 1], e11, T));
          ea = jsc_clamp01(jsc_lin(tb.gp[ipr], ea, tb.gp[ipr + 1], eb, P));
          eps = 1 - (1 - ea) / ps.tp;
          ps.n_ega++;
        }
      }
    }
  }
  return eps;
}

template <int GP, bool DIG, int BLK, int MINB>
__global__ void __launch_bounds__(BLK, MINB) ega_lane_kernel(EgaArgs A) {
  const jsc_dev_model &m = A.m;
  const int nd = m.nd, ng = m.ng;
  const int64_t tid = (int64_t)blockIdx.x * BLK + threadIdx.x;
  const int64_t pc = tid / GP;  // (ray, channel) pair of this lane's group
  const int r = (int)(pc / nd);
  const int d = (int)(pc - (int64_t)r * nd);
  if (r >= A.n_rays) return;  // whole groups leave together
  const int g = (int)(threadIdx.x & (GP - 1));
  const unsigned lane = threadIdx.x & 31;
  const unsigned gbase = lane & ~(unsigned)(GP - 1);
  const unsigned gmask = GP == 32 ? 0xffffffffu : (((1u << GP) - 1u) << gbase);

  const EgaTable tb = ega_table(m, d, g);
  EgaPath ps = ega_path_start();
  double rad = 0, tau = 1;
  const int np = A.nlos[r];
  const int64_t off = A.los_off[r];
  const double *__restrict__ rec = A.pts + off * A.W;
  const double *__restrict__ bc = A.beta_ctm + off * nd + d;
  const double *__restrict__ sp = A.src_pl + off * nd + d;
  const double *__restrict__ ssrc = A.src_sca ? A.src_sca + (size_t)A.sp_off[r] * nd + d : nullptr;

  for (int ip = 0; ip < np; ip++, rec += A.W, bc += nd, sp += nd) {
    const double DS = rec[REC_DS];
    const double eps = ega_lane_eps<DIG>(m, A.single_grid, tb, g, rec, ps);
    ps.tp = ps.tp * (1 - eps);
    // Segment transmittance: the product over emitters in emitter order,
    // as the reference accumulates it (lanes past ng hold eps = 0).
    // All GP factors are fetched first (independent shuffles), then
    // multiplied in emitter order; lanes past ng hold exactly 1.
    const double f = 1 - eps;
    double tau_gas;
    if constexpr (GP <= 8) {
      double fs[GP];
#pragma unroll
      for (int j = 0; j < GP; j++) fs[j] = __shfl_sync(gmask, f, gbase + j);
      tau_gas = fs[0];
#pragma unroll
      for (int j = 1; j < GP; j++) tau_gas *= fs[j];
    } else {  // wider groups: one factor at a time (registers)
      tau_gas = __shfl_sync(gmask, f, gbase);
      for (int j = 1; j < ng; j++) tau_gas *= __shfl_sync(gmask, f, gbase + j);
    }

    const double beta = *bc, src = *sp;
    const double af = rec[REC_AF];
    if (ssrc && af > 0) {
      // scattering point (src/forwardmodel.c:317-363)
      if (tau_gas > 0) {
        const int ia = (int)rec[REC_AI];
        const double be = A.beta[ia * nd + d], bs = A.beta[A.aero_nl * nd + ia * nd + d];
        const double bext = (-1.) * log(tau_gas) / DS + beta + af * be;
        const double e = 1 - exp(-1 * bext * DS);
        const double src_all = ((bext - af * bs) * src + af * bs * *ssrc) / bext;
        rad += tau * e * src_all;
        tau *= exp(-1. * bext * DS);
      }
      ssrc += nd;
    } else if (tau_gas > 0) {
      // clear air, or aerosol/cloud extinction (src/forwardmodel.c:365-389)
      double e;
      if (A.cfg.sca_n == 0 || af == 0) {
        e = 1 - tau_gas * exp(-1. * beta * DS);
      } else {
        const int ia = (int)rec[REC_AI];
        const double bx = A.beta[(A.cfg.sca_ext_beta_a ? 2 : 0) * A.aero_nl * nd + ia * nd + d];
        e = 1 - tau_gas * exp(-1. * (beta + af * bx) * DS);
      }
      rad += src * e * tau;
      tau *= (1 - e);
    }
  }
  if (DIG) {
    // per-channel digest: fold of the per-emitter digests in emitter order
    unsigned long long dd = 0;
    for (int j = 0; j < ng; j++) dd = dd * 1000003ull + __shfl_sync(gmask, ps.dig, gbase + j);
    ps.dig = dd;
  }
  if (g == 0) {
    const double ts = A.tsurf[r];
    if (ts > 0) {
      const int its = planck_index(ts);
      rad += planck_src(m, d, its, ts) * tau;
    }
    A.rad[(size_t)r * nd + d] = rad;
    A.tau[(size_t)r * nd + d] = tau;
    if (DIG) A.digest[(size_t)r * nd + d] = ps.dig;
  }
  const unsigned mask = __activemask();
  const unsigned tot = __reduce_add_sync(mask, ps.n_ega);
  if (lane == (unsigned)(__ffs(mask) - 1)) atomicAdd(&A.counters[1], (unsigned long long)tot);
}

// Warp-level barrier of the NT threads of a block (barrier 1): the emitter
// warps and the transfer warp of ega_ray_kernel reach it from different
// code paths, which a named barrier with an explicit count allows.
__device__ __forceinline__ void ray_barrier(int nt) {
  asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
}

// Radiative-transfer step of one (ray, channel) at one LOS point rec, from
// the point's gas transmittance (the emitters' factors multiplied in
// emitter order), its continuum extinction beta and Planck source src
// (src/forwardmodel.c:302-399); ssrc walks the ray's scattering sources.
__device__ __forceinline__ void rt_point(const EgaArgs &A, int d, int nd,
                                         const double *__restrict__ rec, double tau_gas,
                                         double beta, double src,
                                         const double *__restrict__ &ssrc, double &rad,
                                         double &tau) {
  const double DS = rec[REC_DS];
  const double af = rec[REC_AF];
  if (ssrc && af > 0) {
    // scattering point (src/forwardmodel.c:317-363)
    if (tau_gas > 0) {
      const int ia = (int)rec[REC_AI];
      const double be = A.beta[ia * nd + d], bs = A.beta[A.aero_nl * nd + ia * nd + d];
      const double bext = (-1.) * log(tau_gas) / DS + beta + af * be;
      const double e = 1 - exp(-1 * bext * DS);
      const double src_all = ((bext - af * bs) * src + af * bs * *ssrc) / bext;
      rad += tau * e * src_all;
      tau *= exp(-1. * bext * DS);
    }
    ssrc += nd;
  } else if (tau_gas > 0) {
    // clear air, or aerosol/cloud extinction (src/forwardmodel.c:365-389)
    double e;
    if (A.cfg.sca_n == 0 || af == 0) {
      e = 1 - tau_gas * exp(-1. * beta * DS);
    } else {
      const int ia = (int)rec[REC_AI];
      const double bx = A.beta[(A.cfg.sca_ext_beta_a ? 2 : 0) * A.aero_nl * nd + ia * nd + d];
      e = 1 - tau_gas * exp(-1. * (beta + af * bx) * DS);
    }
    rad += src * e * tau;
    tau *= (1 - e);
  }
}

// Tile and channel of a ray-tile block: tile-major (ORD 0, the blocks of
// one tile side by side) or channel-major (ORD 1, the blocks of one
// channel side by side, so that the blocks resident at a time read the
// tables of few channels).
template <int ORD>
__device__ __forceinline__ void ray_block(int n_rays, int nd, int *tile, int *d) {
  if (ORD == 0) {
    *tile = (int)(blockIdx.x / (unsigned)nd);
    *d = (int)(blockIdx.x - (unsigned)*tile * nd);
  } else {
    const unsigned nt = (unsigned)((n_rays + 31) / 32);
    *d = (int)(blockIdx.x / nt);
    *tile = (int)(blockIdx.x - (unsigned)*d * nt);
  }
}

// The EGA + radiative-transfer kernel with lanes over rays: a block takes
// a tile of 32 rays (ordered so that rays of one profile and similar
// geometry sit side by side) and one channel.  Warp g < NGW evaluates
// emitter g's EGA for the tile's 32 rays at one LOS point after another,
// so the lanes of a warp read the same (channel, emitter) table at nearby
// (p, T) rows and intervals; warp NGW runs the radiative-transfer step one
// point behind, from the emitters' transmittance factors in shared memory
// (two buffers, one barrier per point), multiplying them in emitter order
// as the reference does (src/forwardmodel.c:302-399).
template <int NGW, bool DIG, int MINB, int ORD>
__global__ void __launch_bounds__(32 * (NGW + 1), MINB) ega_ray_kernel(EgaArgs A) {
  constexpr int NT = 32 * (NGW + 1);
  __shared__ double sf[2][NGW][32];
  __shared__ unsigned long long sdig[DIG ? NGW : 1][32];
  const jsc_dev_model &m = A.m;
  const int nd = m.nd, ng = m.ng;
  int tile, d;
  ray_block<ORD>(A.n_rays, nd, &tile, &d);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = tile * 32 + lane;
  const int r = slot < A.n_rays ? A.order[slot] : -1;
  const int np = r >= 0 ? A.nlos[r] : 0;
  // every warp of the block computes the same npmax, so every warp takes
  // the same number of barriers
  int npmax = np;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) npmax = max(npmax, __shfl_xor_sync(0xffffffffu, npmax, o));
  const int64_t off = r >= 0 ? A.los_off[r] : 0;

  if (w < NGW) {
    // emitter warp: the EGA of emitter w for the tile's rays
    const EgaTable tb = ega_table(m, d, w);
    EgaPath ps = ega_path_start();
    const double *__restrict__ rec = A.pts + off * A.W;
    for (int ip = 0; ip < npmax; ip++, rec += A.W) {
      double f = 1;
      if (ip < np) {
        const double eps = ega_lane_eps<DIG>(m, A.single_grid, tb, w, rec, ps);
        ps.tp = ps.tp * (1 - eps);
        f = 1 - eps;
      }
      sf[ip & 1][w][lane] = f;
      ray_barrier(NT);
    }
    if (DIG) sdig[w][lane] = ps.dig;
    const unsigned tot = __reduce_add_sync(0xffffffffu, ps.n_ega);
    if (lane == 0 && tot) atomicAdd(&A.counters[1], (unsigned long long)tot);
    if (DIG) ray_barrier(NT);
    return;
  }

  // transfer warp: the radiance of (ray, channel d) one point behind
  double rad = 0, tau = 1;
  const double *__restrict__ rec = A.pts + off * A.W;
  const double *__restrict__ bc = A.beta_ctm + off * nd + d;
  const double *__restrict__ sp = A.src_pl + off * nd + d;
  const double *__restrict__ ssrc =
      (A.src_sca && r >= 0) ? A.src_sca + (size_t)A.sp_off[r] * nd + d : nullptr;
  for (int ip = 0; ip < npmax; ip++) {
    ray_barrier(NT);  // the factors of point ip are in sf[ip & 1]
    if (ip >= np) continue;
    double tau_gas = sf[ip & 1][0][lane];
    for (int j = 1; j < ng; j++) tau_gas *= sf[ip & 1][j][lane];
    rt_point(A, d, nd, rec, tau_gas, *bc, *sp, ssrc, rad, tau);
    rec += A.W;
    bc += nd;
    sp += nd;
  }
  if (DIG) ray_barrier(NT);  // the emitter warps' digests are in sdig
  if (r < 0) return;
  const double ts = A.tsurf[r];
  if (ts > 0) {
    const int its = planck_index(ts);
    rad += planck_src(m, d, its, ts) * tau;
  }
  A.rad[(size_t)r * nd + d] = rad;
  A.tau[(size_t)r * nd + d] = tau;
  if (DIG) {
    // per-channel digest: fold of the per-emitter digests in emitter order
    unsigned long long dd = 0;
    for (int j = 0; j < ng; j++) dd = dd * 1000003ull + sdig[j][lane];
    A.digest[(size_t)r * nd + d] = dd;
  }
}

// The same tile of 32 rays and one channel without a transfer warp: the
// NGW emitter warps take the radiative-transfer step in turn, warp
// ip mod NGW at LOS point ip right after the point's barrier, with the
// running radiance, transmittance and scattering-source position of the
// tile's rays in shared memory.  The next point's barrier orders one step
// after the other (the warp of step ip reaches barrier ip + 1 only after
// it), and the factor buffer of point ip is rewritten only after barrier
// ip + 1.  Every register of the block goes to EGA warps.
template <int NGW, bool DIG, int MINB, int ORD>
__global__ void __launch_bounds__(32 * NGW, MINB) ega_ray_rot_kernel(EgaArgs A) {
  constexpr int NT = 32 * NGW;
  __shared__ double sf[2][NGW][32];
  __shared__ double srad[32], stau[32];
  __shared__ int ssca[32];
  __shared__ unsigned long long sdig[DIG ? NGW : 1][32];
  const jsc_dev_model &m = A.m;
  const int nd = m.nd, ng = m.ng;
  int tile, d;
  ray_block<ORD>(A.n_rays, nd, &tile, &d);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int slot = tile * 32 + lane;
  const int r = slot < A.n_rays ? A.order[slot] : -1;
  const int np = r >= 0 ? A.nlos[r] : 0;
  int npmax = np;  // the same in every warp: every warp takes npmax + 1 barriers
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) npmax = max(npmax, __shfl_xor_sync(0xffffffffu, npmax, o));
  const int64_t off = r >= 0 ? A.los_off[r] : 0;
  if (w == 0) {
    srad[lane] = 0;
    stau[lane] = 1;
    ssca[lane] = 0;
  }
  const EgaTable tb = ega_table(m, d, w);
  EgaPath ps = ega_path_start();
  const double *__restrict__ rec = A.pts + off * A.W;
  const bool sca = A.src_sca && r >= 0;
  int turn = 0;  // ip mod NGW
  for (int ip = 0; ip < npmax; ip++, rec += A.W) {
    double f = 1;
    if (ip < np) {
      const double eps = ega_lane_eps<DIG>(m, A.single_grid, tb, w, rec, ps);
      ps.tp = ps.tp * (1 - eps);
      f = 1 - eps;
    }
    sf[ip & 1][w][lane] = f;
    ray_barrier(NT);  // the factors of point ip are in sf[ip & 1]
    if (w == turn && ip < np) {
      double tau_gas = sf[ip & 1][0][lane];
      for (int j = 1; j < ng; j++) tau_gas *= sf[ip & 1][j][lane];
      double rad = srad[lane], tau = stau[lane];
      const int isp = ssca[lane];
      const double *__restrict__ ssrc =
          sca ? A.src_sca + ((size_t)A.sp_off[r] + isp) * nd + d : nullptr;
      const double *__restrict__ s0 = ssrc;
      const size_t pc = (size_t)(off + ip) * nd + d;
      rt_point(A, d, nd, rec, tau_gas, A.beta_ctm[pc], A.src_pl[pc], ssrc, rad, tau);
      srad[lane] = rad;
      stau[lane] = tau;
      if (ssrc != s0) ssca[lane] = isp + 1;
    }
    turn = turn + 1 == NGW ? 0 : turn + 1;
  }
  if (DIG) sdig[w][lane] = ps.dig;
  const unsigned tot = __reduce_add_sync(0xffffffffu, ps.n_ega);
  if (lane == 0 && tot) atomicAdd(&A.counters[1], (unsigned long long)tot);
  ray_barrier(NT);  // the last step and the digests are in shared memory
  if (w != 0 || r < 0) return;
  double rad = srad[lane];
  const double tau = stau[lane];
  const double ts = A.tsurf[r];
  if (ts > 0) {
    const int its = planck_index(ts);
    rad += planck_src(m, d, its, ts) * tau;
  }
  A.rad[(size_t)r * nd + d] = rad;
  A.tau[(size_t)r * nd + d] = tau;
  if (DIG) {
    unsigned long long dd = 0;
    for (int j = 0; j < ng; j++) dd = dd * 1000003ull + sdig[j][lane];
    A.digest[(size_t)r * nd + d] = dd;
  }
}

// Ray-tile variants v: 0-2 with a transfer warp, (resident blocks per SM
// at 8 emitters, block order) = (3, tile-major), (4, tile-major), (4,
// channel-major); 3-6 with the step taken in turn: (4, tile), (5, tile),
// (4, channel), (5, channel).  Other emitter counts keep the threads per
// SM of 8 emitters, i.e. the register budget per thread.
template <int NGW, bool DIG, int MINB8, int ORD>
static void ega_ray_tr(const EgaArgs &ea, unsigned blocks, cudaStream_t s) {
  constexpr int MB = MINB8 * 9 / (NGW + 1) > 1 ? MINB8 * 9 / (NGW + 1) : 1;
  ega_ray_kernel<NGW, DIG, MB, ORD><<<blocks, 32 * (NGW + 1), 0, s>>>(ea);
}

template <int NGW, bool DIG, int MINB8, int ORD>
static void ega_ray_rot(const EgaArgs &ea, unsigned blocks, cudaStream_t s) {
  constexpr int MB = MINB8 * 8 / NGW > 1 ? MINB8 * 8 / NGW : 1;
  ega_ray_rot_kernel<NGW, DIG, MB, ORD><<<blocks, 32 * NGW, 0, s>>>(ea);
}

template <int NGW, bool DIG>
static void ega_ray_launch(const EgaArgs &ea, int v, cudaStream_t s) {
  const unsigned blocks = (unsigned)(((int64_t)ea.n_rays + 31) / 32 * ea.m.nd);
  switch (v) {
    case 0: ega_ray_tr<NGW, DIG, 3, 0>(ea, blocks, s); break;
    case 1: ega_ray_tr<NGW, DIG, 4, 0>(ea, blocks, s); break;
    case 2: ega_ray_tr<NGW, DIG, 4, 1>(ea, blocks, s); break;
    case 3: ega_ray_rot<NGW, DIG, 4, 0>(ea, blocks, s); break;
    case 4: ega_ray_rot<NGW, DIG, 5, 0>(ea, blocks, s); break;
    case 5: ega_ray_rot<NGW, DIG, 4, 1>(ea, blocks, s); break;
    default: ega_ray_rot<NGW, DIG, 5, 1>(ea, blocks, s); break;
  }
}

template <int NGW>
static void ega_ray_variant(const EgaArgs &ea, int v, bool dig, cudaStream_t s) {
  if (dig) ega_ray_launch<NGW, true>(ea, v, s);
  else ega_ray_launch<NGW, false>(ea, v, s);
}

// Launch variants of ega_lane_kernel: (threads per block, minimum resident
// blocks per SM), each with and without index digests.
template <int GP, bool DIG>
static void ega_lane_launch(const EgaArgs &ea, int v, cudaStream_t s) {
  const int64_t threads = (int64_t)ea.n_rays * ea.m.nd * GP;
  switch (v) {
    case 1: ega_lane_kernel<GP, DIG, 128, 8><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(ea); break;
    case 2: ega_lane_kernel<GP, DIG, 256, 4><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(ea); break;
    case 3: ega_lane_kernel<GP, DIG, 256, 5><<<(unsigned)((threads + 255) / 256), 256, 0, s>>>(ea); break;
    case 4: ega_lane_kernel<GP, DIG, 512, 2><<<(unsigned)((threads + 511) / 512), 512, 0, s>>>(ea); break;
    default: ega_lane_kernel<GP, DIG, 128, 12><<<(unsigned)((threads + 127) / 128), 128, 0, s>>>(ea); break;
  }
}

template <int GP>
static void ega_lane_variant(const EgaArgs &ea, int v, bool dig, cudaStream_t s) {
  if (dig) ega_lane_launch<GP, true>(ea, v, s);
  else ega_lane_launch<GP, false>(ea, v, s);
}

// Launchers (ega_lane_s.cu: up to 4 emitters, ega_lane_l.cu: more and the
// continuum kernel): lanes per group from the emitter count.
void jsc_ega_lane_launch_s(const EgaArgs &ea, int v, bool dig, cudaStream_t s);
void jsc_ega_lane_launch_l(const EgaArgs &ea, int v, bool dig, cudaStream_t s);
void jsc_ctm_src_launch(const CtmArgs &ca, cudaStream_t s);
// Ray-tile kernel (ega_ray.cu) for up to 16 emitters, and the ray order it
// reads (sorted keys: profile, surface hit, LOS point count, tangent
// altitude).
void jsc_ega_ray_launch(const EgaArgs &ea, int v, bool dig, cudaStream_t s);
int jsc_ray_order(int n_rays, const int *ray_atm, const int *nlos, const double *tsurf,
                  const double *tpz, unsigned long long *keys, int *order, void *tmp,
                  size_t tmp_bytes, cudaStream_t s);
size_t jsc_ray_order_tmp_bytes(int max_rays);
#define JSC_LANE_VARIANTS 5
