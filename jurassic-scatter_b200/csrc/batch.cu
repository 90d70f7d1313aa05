// Batches: device buffers for many rays over many atmospheric profiles, and
// the launch sequence of one forward model over them.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "kernels.cuh"
#include "ega_kernel.cuh"
#include "ega_lane.cuh"
#include "scatter.cuh"
#include "surrogate.h"

static int sca_alpha(double *alpha, int nalpha);
static int map_status(unsigned st);

static void batch_free_los(jsc_batch *b) {
  cudaFree(b->d_geo);
  cudaFree(b->d_pts);
  cudaFree(b->d_ctm);
  cudaFree(b->d_srcp);
  b->d_geo = b->d_pts = b->d_ctm = b->d_srcp = nullptr;
}

static int batch_alloc_los(jsc_batch *b, int64_t max_seg) {
  batch_free_los(b);
  int st;
  if ((st = jsc_dmalloc(&b->d_geo, (size_t)max_seg * 4))) return st;
  if ((st = jsc_dmalloc(&b->d_pts, (size_t)max_seg * b->W))) return st;
  if ((st = jsc_dmalloc(&b->d_ctm, (size_t)max_seg * b->cfg.nd))) return st;
  if ((st = jsc_dmalloc(&b->d_srcp, (size_t)max_seg * b->cfg.nd))) return st;
  b->max_seg = max_seg;
  return JSC_OK;
}

extern "C" void jsc_batch_destroy(jsc_batch *b) {
  if (!b) return;
  cudaFree(b->d_atm_off);
  cudaFree(b->d_z);
  cudaFree(b->d_lon);
  cudaFree(b->d_lat);
  cudaFree(b->d_psurf);
  cudaFree(b->d_p_in);
  cudaFree(b->d_t);
  cudaFree(b->d_q);
  cudaFree(b->d_k);
  cudaFree(b->d_p);
  cudaFree(b->d_zmin);
  cudaFree(b->d_zmax);
  cudaFree(b->d_ray_atm);
  cudaFree(b->d_ray);
  cudaFree(b->d_nlos);
  cudaFree(b->d_los_off);
  batch_free_los(b);
  cudaFree(b->d_tsurf);
  cudaFree(b->d_tp);
  cudaFree(b->d_rkeys);
  cudaFree(b->d_rorder);
  cudaFree(b->d_rtmp);
  cudaFree(b->d_rad);
  cudaFree(b->d_tau);
  cudaFree(b->d_status);
  cudaFree(b->d_counters);
  cudaFree(b->d_digest);
  cudaFree(b->d_scan);
  cudaFree(b->d_sp_listed);
  cudaFree(b->d_live);
  cudaFree(b->d_qhead);
  cudaFree(b->d_aero);
  cudaFree(b->d_beta);
  cudaFree(b->d_phase);
  cudaFree(b->d_nlos_b);
  cudaFree(b->d_los_off_b);
  cudaFree(b->d_geo_b);
  cudaFree(b->d_pts_b);
  cudaFree(b->d_nsp);
  cudaFree(b->d_sp_off);
  cudaFree(b->d_sp);
  cudaFree(b->d_sp_atm);
  cudaFree(b->d_src);
  cudaFree(b->d_theta2);
  cudaFree(b->d_planck_sun);
  jsc_batch_destroy(b->child);
  jsc_batch_destroy(b->sun_child);
  cudaFree(b->d_feat);
  cudaFree(b->d_mark);
  cudaFree(b->d_idx);
  cudaFree(b->d_sp_sub);
  cudaFree(b->d_atm_sub);
  cudaFree(b->d_src_sub);
  free(b->h_aero);
  free(b->ctl);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->h_status) cudaFreeHost(b->h_status);
  if (b->h_total) cudaFreeHost(b->h_total);
  for (int i = 0; i < 2 * JSC_T_N; i++)
    if (b->ev[i]) cudaEventDestroy(b->ev[i]);
  free(b);
}

extern "C" int jsc_batch_create(jsc_model *m, const ctl_t *ctl, int max_atm,
                                int max_levels, int max_rays, int64_t max_seg,
                                jsc_batch **out) {
  if (!m || !ctl || !out || max_atm < 1 || max_levels < 2 || max_rays < 1) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_create: invalid arguments");
    return JSC_ERR_ARG;
  }
  *out = nullptr;
  if (ctl->ng != m->ng || ctl->nd != m->nd || ctl->nw != m->nw) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_create: ctl does not match the model");
    return JSC_ERR_ARG;
  }
  if (ctl->ip < 1 || ctl->ip > 3) {
    jsc_set_error(JSC_ERR_ARG, "unknown interpolation method IP=%d", ctl->ip);
    return JSC_ERR_ARG;
  }
  if (ctl->ip == 3 && !(ctl->cz > 0 && ctl->cx > 0)) {
    jsc_set_error(JSC_ERR_ARG, "IP=3 needs positive influence lengths CZ, CX");
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaSetDevice(m->device));
  jsc_batch *b = (jsc_batch *)calloc(1, sizeof(jsc_batch));
  if (!b) return JSC_ERR_NOMEM;
  b->m = m;
  jsc_run_cfg &c = b->cfg;
  c.ng = ctl->ng;
  c.nd = ctl->nd;
  c.nw = ctl->nw;
  c.ctm_co2 = ctl->ctm_co2;
  c.ctm_h2o = ctl->ctm_h2o;
  c.ctm_n2 = ctl->ctm_n2;
  c.ctm_o2 = ctl->ctm_o2;
  c.refrac = ctl->refrac;
  c.rayds = ctl->rayds;
  c.raydz = ctl->raydz;
  c.hydz = ctl->hydz;
  c.sca_n = ctl->sca_n;
  c.sca_mult = ctl->sca_mult;
  c.sca_ext_beta_a = strcmp(ctl->sca_ext, "beta_a") == 0;
  c.transs = ctl->transs;
  b->max_atm = max_atm;
  b->max_levels = max_levels;
  b->max_rays = max_rays;
  b->W = JSC_REC_W(ctl->nw, ctl->ng);
  const int ng = ctl->ng > 0 ? ctl->ng : 1, nw = ctl->nw > 0 ? ctl->nw : 1;
  int st = JSC_OK;
  st = st ? st : jsc_dmalloc(&b->d_atm_off, (size_t)max_atm + 1);
  st = st ? st : jsc_dmalloc(&b->d_z, (size_t)max_levels);
  st = st ? st : jsc_dmalloc(&b->d_lon, (size_t)max_levels);
  st = st ? st : jsc_dmalloc(&b->d_lat, (size_t)max_levels);
  b->ip = ctl->ip;
  b->cz = ctl->cz;
  b->cx = ctl->cx;
  if (ctl->ip != 1)
    st = st ? st : jsc_dmalloc(&b->d_psurf, 3 * (size_t)(max_levels > max_atm ? max_levels : max_atm));
  st = st ? st : jsc_dmalloc(&b->d_p_in, (size_t)max_levels);
  st = st ? st : jsc_dmalloc(&b->d_t, (size_t)max_levels);
  st = st ? st : jsc_dmalloc(&b->d_q, (size_t)max_levels * ng);
  st = st ? st : jsc_dmalloc(&b->d_k, (size_t)max_levels * nw);
  st = st ? st : jsc_dmalloc(&b->d_p, (size_t)max_levels);
  st = st ? st : jsc_dmalloc(&b->d_zmin, (size_t)max_atm);
  st = st ? st : jsc_dmalloc(&b->d_zmax, (size_t)max_atm);
  st = st ? st : jsc_dmalloc(&b->d_ray_atm, (size_t)max_rays);
  st = st ? st : jsc_dmalloc(&b->d_ray, (size_t)max_rays * 9);
  st = st ? st : jsc_dmalloc(&b->d_nlos, (size_t)max_rays);
  st = st ? st : jsc_dmalloc(&b->d_los_off, (size_t)max_rays + 1);
  st = st ? st : jsc_dmalloc(&b->d_tsurf, (size_t)max_rays);
  st = st ? st : jsc_dmalloc(&b->d_tp, (size_t)max_rays * 3);
  st = st ? st : jsc_dmalloc(&b->d_rkeys, (size_t)max_rays * 2);
  st = st ? st : jsc_dmalloc(&b->d_rorder, (size_t)max_rays * 2);
  if (!st) {
    b->rtmp_bytes = jsc_ray_order_tmp_bytes(max_rays);
    if (cudaMalloc(&b->d_rtmp, b->rtmp_bytes ? b->rtmp_bytes : 16) != cudaSuccess) {
      jsc_set_error(JSC_ERR_NOMEM, "device allocation of %zu bytes", b->rtmp_bytes);
      st = JSC_ERR_NOMEM;
    }
  }
  st = st ? st : jsc_dmalloc(&b->d_rad, (size_t)max_rays * ctl->nd);
  st = st ? st : jsc_dmalloc(&b->d_tau, (size_t)max_rays * ctl->nd);
  st = st ? st : jsc_dmalloc(&b->d_status, 1);
  st = st ? st : jsc_dmalloc(&b->d_counters, 2);
  if (!st) st = batch_alloc_los(b, max_seg > 0 ? max_seg : (int64_t)max_rays * 512);
  b->scan_tiles = (max_rays + JSC_SCAN_TILE - 1) / JSC_SCAN_TILE + 1;
  st = st ? st : jsc_dmalloc(&b->d_scan, (size_t)b->scan_tiles + 1);
  b->wait_budget = JSC_WAIT_BUDGET;
  b->ega_variant = -1;
  for (int v = 0; v < 32; v++) b->ega_variant_ms[v] = -1;
  b->depth = ctl->sca_n > 0 ? ctl->sca_mult : 0;
  b->nalpha = JSC_NALPHA_REF;
  sca_alpha(b->alpha, b->nalpha);
  b->ctl = (ctl_t *)malloc(sizeof(ctl_t));
  if (!b->ctl) st = st ? st : JSC_ERR_NOMEM;
  else memcpy(b->ctl, ctl, sizeof(ctl_t));
  if (!st && cudaMallocHost((void **)&b->h_total, sizeof(int64_t)) != cudaSuccess) {
    jsc_set_error(JSC_ERR_NOMEM, "pinned host allocation");
    st = JSC_ERR_NOMEM;
  }
  for (int i = 0; i < 2 * JSC_T_N && !st; i++)
    if (cudaEventCreate(&b->ev[i]) != cudaSuccess) st = JSC_ERR_CUDA;
  if (st) {
    jsc_batch_destroy(b);
    return st;
  }
  *out = b;
  return JSC_OK;
}

// Zenith angles of the secondary pencils: 0, a Fibonacci-spaced fan down to
// the horizon, 1-degree steps from 83 to 90 degrees, the mirrored fan up,
// and pi (src/scatter.c:695-715 for 28 pencils; any even count from 10 to
// 28 gives increasing angles the same way).
static int sca_alpha(double *alpha, int nalpha) {
  if (nalpha < 10 || nalpha > JSC_NALPHA_REF || (nalpha & 1)) return JSC_ERR_ARG;
  int n1 = 1, n2 = 2;
  double midang = 83, up = 92, down = 81, step = 1 + 2;
  alpha[0] = 0;
  for (int ir = nalpha / 2 - 4; ir < nalpha / 2 + 4; ++ir) {
    alpha[ir] = midang * M_PI / 180.;
    midang++;
  }
  for (int ir = 0; ir < nalpha / 2 - 5; ++ir) {
    alpha[nalpha / 2 + ir + 4] = up * M_PI / 180.;
    alpha[nalpha / 2 - ir - 5] = down * M_PI / 180.;
    up += step;
    down -= step;
    if (step < 13) {
      step = (double)n1 + (double)n2;
      n1 = n2;
      n2 = (int)step;
    }
  }
  alpha[nalpha - 1] = M_PI;
  for (int i = 0; i + 1 < nalpha; i++)
    if (!(alpha[i] < alpha[i + 1])) return JSC_ERR_ARG;
  return JSC_OK;
}

extern "C" int jsc_batch_set_nalpha(jsc_batch *b, int nalpha) {
  if (!b || sca_alpha(b->alpha, nalpha)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_nalpha: %d secondary pencils (even, 10..%d)",
                  nalpha, JSC_NALPHA_REF);
    if (b) sca_alpha(b->alpha, b->nalpha);
    return JSC_ERR_ARG;
  }
  b->nalpha = nalpha;
  for (int d = 0; d <= JSC_MAX_DEPTH; d++) b->nalpha_at[d] = 0;
  // child batches are sized per pencil count: rebuild on the next run
  jsc_batch_destroy(b->child);
  b->child = nullptr;
  return JSC_OK;
}

extern "C" int jsc_batch_set_nalpha_depth(jsc_batch *b, int depth, int nalpha) {
  double alpha[32];
  if (!b || depth < 1 || depth > JSC_MAX_DEPTH || depth > b->depth || sca_alpha(alpha, nalpha)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_nalpha_depth: depth %d (1..%d) with %d pencils "
                  "(even, 10..%d)", depth, b ? b->depth : 0, nalpha, JSC_NALPHA_REF);
    return JSC_ERR_ARG;
  }
  b->nalpha_at[depth] = nalpha;
  if (depth == b->depth) {
    b->nalpha = nalpha;
    memcpy(b->alpha, alpha, sizeof(alpha));
  }
  // child batches are sized per pencil count: rebuild on the next run
  jsc_batch_destroy(b->child);
  b->child = nullptr;
  return JSC_OK;
}

static int cmp_desc(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

extern "C" int jsc_batch_set_aero(jsc_batch *b, const aero_t *aero) {
  if (!b || !aero || aero->nl < 0 || aero->nl > NLMAX) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_aero: invalid aerosol layers");
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  const int nl = aero->nl, nd = b->cfg.nd;
  // Layer edges +-5 m and transition sampling altitudes, top down
  // (src/lineofsight.c:210-244).
  const double eps = 0.005;
  double *alti = (double *)malloc(sizeof(double) * (4 * NLMAX + 2 * 4096));
  int jl = 0;
  if (!alti) return JSC_ERR_NOMEM;
  for (int il = 0; il < nl; il++) {
    alti[jl] = aero->top[il] + eps;
    alti[jl + 1] = aero->top[il] - eps;
    alti[jl + 2] = aero->bottom[il] + eps;
    alti[jl + 3] = aero->bottom[il] - eps;
    jl += 4;
    if (aero->trans[il] > b->cfg.transs) {
      const double tt = aero->trans[il] / b->cfg.transs;
      alti[jl] = aero->top[il] + aero->trans[il] + eps;
      alti[jl + 1] = aero->top[il] + aero->trans[il] - eps;
      alti[jl + 2] = aero->bottom[il] - aero->trans[il] + eps;
      alti[jl + 3] = aero->bottom[il] - aero->trans[il] - eps;
      jl += 4;
      for (int it = 1; it < (int)tt; it++) {
        if (jl + 2 > 4 * NLMAX + 2 * 4096) {
          free(alti);
          jsc_set_error(JSC_ERR_ARG, "too many transition-layer samples");
          return JSC_ERR_ARG;
        }
        alti[jl++] = aero->top[il] + aero->trans[il] - eps - it * b->cfg.transs;
        alti[jl++] = aero->bottom[il] - aero->trans[il] + eps + it * b->cfg.transs;
      }
    }
  }
  qsort(alti, (size_t)jl, sizeof(double), cmp_desc);
  double amax = jl ? alti[0] : 0, amin = jl ? alti[0] : 0;
  for (int i = 0; i < jl; i++) {
    if (alti[i] > amax) amax = alti[i];
    if (alti[i] < amin) amin = alti[i];
  }
  const size_t nh = 3 * NLMAX + (size_t)jl;
  double *h = (double *)calloc(nh > 0 ? nh : 1, sizeof(double));
  double *beta = (double *)calloc((size_t)3 * (nl > 0 ? nl : 1) * nd, sizeof(double));
  double *phase = (double *)calloc((size_t)(nl > 0 ? nl : 1) * nd * NTHETA, sizeof(double));
  if (!h || !beta || !phase) {
    free(alti); free(h); free(beta); free(phase);
    return JSC_ERR_NOMEM;
  }
  for (int il = 0; il < nl; il++) {
    h[il] = aero->top[il];
    h[NLMAX + il] = aero->bottom[il];
    h[2 * NLMAX + il] = aero->trans[il];
    for (int id = 0; id < nd; id++) {
      beta[(size_t)il * nd + id] = aero->beta_e[il][id];
      beta[(size_t)(nl + il) * nd + id] = aero->beta_s[il][id];
      beta[(size_t)(2 * nl + il) * nd + id] = aero->beta_a[il][id];
      for (int ia = 0; ia < NTHETA; ia++)
        phase[((size_t)il * nd + id) * NTHETA + ia] = aero->p[il][id][ia];
    }
  }
  memcpy(h + 3 * NLMAX, alti, sizeof(double) * (size_t)jl);
  cudaFree(b->d_aero);
  cudaFree(b->d_beta);
  cudaFree(b->d_phase);
  b->d_aero = nullptr;
  b->d_beta = b->d_phase = nullptr;
  int st = jsc_dmalloc(&b->d_aero, nh);
  if (!st) st = jsc_dmalloc(&b->d_beta, (size_t)3 * (nl > 0 ? nl : 1) * nd);
  if (!st) st = jsc_dmalloc(&b->d_phase, (size_t)(nl > 0 ? nl : 1) * nd * NTHETA);
  if (!st && cudaMemcpy(b->d_aero, h, nh * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) st = JSC_ERR_CUDA;
  if (!st && cudaMemcpy(b->d_beta, beta, (size_t)3 * (nl > 0 ? nl : 1) * nd * sizeof(double),
                        cudaMemcpyHostToDevice) != cudaSuccess) st = JSC_ERR_CUDA;
  if (!st && cudaMemcpy(b->d_phase, phase, (size_t)(nl > 0 ? nl : 1) * nd * NTHETA * sizeof(double),
                        cudaMemcpyHostToDevice) != cudaSuccess) st = JSC_ERR_CUDA;
  free(alti); free(h); free(beta); free(phase);
  if (st) {
    jsc_set_error(st, "jsc_batch_set_aero: device upload failed");
    return st;
  }
  if (!b->h_aero && !(b->h_aero = (aero_t *)malloc(sizeof(aero_t)))) return JSC_ERR_NOMEM;
  if (b->h_aero != aero) memcpy(b->h_aero, aero, sizeof(aero_t));
  b->aero_nl = nl;
  b->n_alti = jl;
  b->altimax = amax;
  b->altimin = amin;
  // child batches (secondary and solar pencils) see the same layers
  for (jsc_batch *c : {b->child, b->sun_child})
    if (c && (st = jsc_batch_set_aero(c, aero))) return st;
  if (!b->d_nlos_b) {
    if ((st = jsc_dmalloc(&b->d_nlos_b, (size_t)b->max_rays))) return st;
    if ((st = jsc_dmalloc(&b->d_los_off_b, (size_t)b->max_rays + 1))) return st;
  }
  return JSC_OK;
}

static int batch_alloc_los_b(jsc_batch *b, int64_t max_seg) {
  cudaFree(b->d_geo_b);
  cudaFree(b->d_pts_b);
  b->d_geo_b = b->d_pts_b = nullptr;
  int st;
  if ((st = jsc_dmalloc(&b->d_geo_b, (size_t)max_seg * 4))) return st;
  if ((st = jsc_dmalloc(&b->d_pts_b, (size_t)max_seg * b->W))) return st;
  b->max_seg_b = max_seg;
  return JSC_OK;
}

#define CPY(dst, src, n, s)                                                  \
  JSC_CUDA_TRY(cudaMemcpyAsync((dst), (src), (size_t)(n) * sizeof(*(src)),   \
                               cudaMemcpyHostToDevice, (cudaStream_t)(s)))

extern "C" int jsc_batch_upload(jsc_batch *b, const jsc_batch_input *in,
                                void *stream) {
  if (!b || !in) return JSC_ERR_ARG;
  const int ng = b->cfg.ng, nw = b->cfg.nw;
  if (in->n_atm < 1 || in->n_atm > b->max_atm || in->n_levels < 2 ||
      in->n_levels > b->max_levels || in->n_rays < 0 || in->n_rays > b->max_rays) {
    jsc_set_error(JSC_ERR_ARG, "batch input exceeds the batch capacity");
    return JSC_ERR_ARG;
  }
  // Validate every index the kernels follow, so no device access leaves its
  // buffer: profile offsets increase and stay inside the level arrays, every
  // profile has two levels or more, every ray names an existing profile.
  if (in->atm_off[0] != 0 || in->atm_off[in->n_atm] != in->n_levels) {
    jsc_set_error(JSC_ERR_ARG, "atm_off must start at 0 and end at n_levels");
    return JSC_ERR_ARG;
  }
  for (int a = 0; a < in->n_atm; a++)
    if (in->atm_off[a + 1] - in->atm_off[a] < 2) {
      jsc_set_error(JSC_ERR_ARG, "profile %d has fewer than 2 levels", a);
      return JSC_ERR_ARG;
    }
  for (int r = 0; r < in->n_rays; r++)
    if (in->ray_atm[r] < 0 || in->ray_atm[r] >= in->n_atm) {
      jsc_set_error(JSC_ERR_ARG, "ray %d names profile %d of %d", r,
                    in->ray_atm[r], in->n_atm);
      return JSC_ERR_ARG;
    }
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  b->n_atm = in->n_atm;
  b->n_levels = in->n_levels;
  b->n_rays = in->n_rays;
  const int nl = in->n_levels, nr = in->n_rays;
  CPY(b->d_atm_off, in->atm_off, in->n_atm + 1, stream);
  CPY(b->d_z, in->z, nl, stream);
  CPY(b->d_lon, in->lon, nl, stream);
  CPY(b->d_lat, in->lat, nl, stream);
  CPY(b->d_p_in, in->p, nl, stream);
  CPY(b->d_t, in->t, nl, stream);
  if (ng > 0) CPY(b->d_q, in->q, (size_t)ng * nl, stream);
  if (nw > 0) CPY(b->d_k, in->k, (size_t)nw * nl, stream);
  if (nr > 0) {
    CPY(b->d_ray_atm, in->ray_atm, nr, stream);
    const double *cols[7] = {in->time, in->obsz, in->obslon, in->obslat,
                             in->vpz, in->vplon, in->vplat};
    for (int i = 0; i < 7; i++) {
      if (cols[i]) {
        CPY(b->d_ray + (size_t)i * nr, cols[i], nr, stream);
      } else {
        JSC_CUDA_TRY(cudaMemsetAsync(b->d_ray + (size_t)i * nr, 0,
                                     (size_t)nr * sizeof(double),
                                     (cudaStream_t)stream));
      }
    }
  }
  return JSC_OK;
}

// Exclusive prefix sum of n counts into out[0..n] (scan_lookback_kernel),
// on the batch's scan scratch (n <= max_rays); waits give up after the
// batch's wait budget with JSC_DEV_ERR_WATCHDOG in its status word.
static int launch_scan(jsc_batch *b, const int *in, int n, int64_t *out, cudaStream_t s) {
  if (n <= 0) {
    JSC_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    return JSC_OK;
  }
  const int tiles = (n + JSC_SCAN_TILE - 1) / JSC_SCAN_TILE;
  if (tiles > b->scan_tiles) {
    jsc_set_error(JSC_ERR_ARG, "scan of %d counts exceeds the batch's %d tiles", n, b->scan_tiles);
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaMemsetAsync(b->d_scan, 0, ((size_t)tiles + 1) * sizeof(unsigned long long), s));
  ScanArgs a;
  a.in = in;
  a.n = n;
  a.out = out;
  a.flags = b->d_scan + 1;
  a.ticket = reinterpret_cast<unsigned *>(b->d_scan);
  a.status = b->d_status;
  a.budget = b->wait_budget;
  a.stall_tile = -1;
  scan_lookback_kernel<<<tiles, JSC_SCAN_THREADS, 0, s>>>(a);
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

extern "C" int jsc_batch_set_wait_budget(jsc_batch *b, unsigned polls) {
  if (!b) return JSC_ERR_ARG;
  b->wait_budget = polls ? polls : JSC_WAIT_BUDGET;
  return JSC_OK;
}

extern "C" int jsc_scan_selftest(int device, int n, unsigned budget, int stall) {
  if (n < 1 || n > (1 << 26)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_scan_selftest: n = %d outside 1..2^26", n);
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaSetDevice(device));
  const int tiles = (n + JSC_SCAN_TILE - 1) / JSC_SCAN_TILE;
  int *d_in = nullptr;
  int64_t *d_out = nullptr;
  unsigned long long *d_scan = nullptr;
  unsigned *d_status = nullptr;
  int st = jsc_dmalloc(&d_in, (size_t)n);
  if (!st) st = jsc_dmalloc(&d_out, (size_t)n + 1);
  if (!st) st = jsc_dmalloc(&d_scan, (size_t)tiles + 1);
  if (!st) st = jsc_dmalloc(&d_status, 1);
  int *h_in = (int *)malloc((size_t)n * sizeof(int));
  int64_t *h_out = (int64_t *)malloc(((size_t)n + 1) * sizeof(int64_t));
  if (!st && (!h_in || !h_out)) st = JSC_ERR_NOMEM;
  cudaStream_t s = nullptr;
  if (!st && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) st = JSC_ERR_CUDA;
  unsigned status = 0;
  if (!st) {
    for (int i = 0; i < n; i++) h_in[i] = (int)((i * 2654435761u) >> 27);  // 0..31
    cudaError_t e = cudaMemcpyAsync(d_in, h_in, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_scan, 0, ((size_t)tiles + 1) * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) {
      ScanArgs a;
      a.in = d_in;
      a.n = n;
      a.out = d_out;
      a.flags = d_scan + 1;
      a.ticket = reinterpret_cast<unsigned *>(d_scan);
      a.status = d_status;
      a.budget = budget ? budget : JSC_WAIT_BUDGET;
      a.stall_tile = stall;
      scan_lookback_kernel<<<tiles, JSC_SCAN_THREADS, 0, s>>>(a);
      jsc_count_launch();
      e = cudaGetLastError();
    }
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_out, d_out, ((size_t)n + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&status, d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
      jsc_set_error(JSC_ERR_CUDA, "jsc_scan_selftest: %s", cudaGetErrorString(e));
      st = JSC_ERR_CUDA;
    }
  }
  if (!st) {
    st = map_status(status);
    if (!st) {
      int64_t run = 0;
      for (int i = 0; i <= n && !st; i++) {
        if (h_out[i] != run) {
          jsc_set_error(JSC_ERR_CUDA, "jsc_scan_selftest: prefix %d is %lld, expected %lld", i,
                        (long long)h_out[i], (long long)run);
          st = JSC_ERR_CUDA;
        }
        if (i < n) run += h_in[i];
      }
    }
  }
  if (s) cudaStreamDestroy(s);
  cudaFree(d_in);
  cudaFree(d_out);
  cudaFree(d_scan);
  cudaFree(d_status);
  free(h_in);
  free(h_out);
  return st;
}

// Launch variants of the EGA + radiative-transfer step.  0-8: ega_rt_kernel,
// a thread per (ray, channel) with all emitters' path state: (threads per
// block, minimum resident blocks per SM, emitter loop rolled); the second
// number sets the register budget, i.e. the trade between occupancy and
// spills, the rolled loop trades registers and instruction-cache footprint
// for local-memory path state.  9-13: ega_lane_kernel, a lane per
// (ray, channel, emitter), after ctm_src_kernel.  14-20: lanes over a
// tile of 32 ordered rays, a warp per emitter, after ctm_src_kernel
// (blk 0 here: the block size follows the emitter count); ray 1:
// ega_ray_kernel with a transfer warp (block 32 (emitter warps + 1)),
// ray 2: ega_ray_rot_kernel, the emitter warps take the transfer step in
// turn (block 32 emitter warps); 16 and 19-20 order the blocks
// channel-major.  More than 16 emitters run the lane variant 13 instead.
// jsc_batch_autotune picks one.
struct EgaVariant { int blk, minb, roll, lane, ray; };
static const EgaVariant kEgaVariants[] = {
    {128, 4, 0, 0, 0}, {128, 6, 0, 0, 0}, {128, 8, 0, 0, 0}, {256, 3, 0, 0, 0},
    {256, 4, 0, 0, 0}, {128, 8, 1, 0, 0}, {128, 12, 1, 0, 0}, {256, 4, 1, 0, 0},
    {256, 6, 1, 0, 0}, {128, 12, 0, 1, 0}, {128, 8, 0, 1, 0}, {256, 4, 0, 1, 0},
    {256, 5, 0, 1, 0}, {512, 2, 0, 1, 0}, {0, 3, 0, 1, 1}, {0, 4, 0, 1, 1},
    {0, 4, 0, 1, 1},   {0, 4, 0, 1, 2},   {0, 5, 0, 1, 2}, {0, 4, 0, 1, 2},
    {0, 5, 0, 1, 2}};
static const int kNumEgaVariants = 21;
static_assert(kNumEgaVariants <= 32, "ega_variant_ms holds 32 timings");
static const int kLaneBase = 9;
static const int kRayBase = 14;

// Emitter warps of the ray-tile kernel for ng emitters (0: not available).
static int ray_warps(int ng) {
  return ng <= 2 ? 2 : ng <= 4 ? 4 : ng <= 8 ? 8 : ng <= 16 ? 16 : 0;
}
// Default launch variant of clear-air runs: the ray-tile kernel with the
// transfer step taken in turn (422 ms against 631 ms for the fastest lane
// variant and 716 ms for the thread-per-channel variant 6 on 100k rays,
// 8 emitters, 64 channels).
static const int kEgaDefault = 17;

// Default launch variant of runs with aerosol/cloud layers (the scattering
// path and its child batches): the same ray-tile kernel (819 ms per plain
// single-scattering step of 4000 limb rays, 16 channels, 2 emitters,
// against 847 ms for the lane variant 10).
static const int kScatterDefault = 17;

// The variant a run of b launches (-1 resolves to the default for its
// configuration).
static int run_variant(const jsc_batch *b) {
  if (b->ega_variant >= 0 && b->ega_variant < kNumEgaVariants) return b->ega_variant;
  return b->cfg.sca_n > 0 ? kScatterDefault : kEgaDefault;
}

static bool lane_variant(int variant) {
  const int v = (variant >= 0 && variant < kNumEgaVariants) ? variant : kEgaDefault;
  return kEgaVariants[v].lane != 0;
}

static int launch_ega(const EgaArgs &ea, int nr, int ndp, int ng, int variant,
                      cudaStream_t s) {
  const int64_t threads = (int64_t)nr * ndp;
  const unsigned g128 = (unsigned)((threads + 127) / 128);
  const unsigned g256 = (unsigned)((threads + 255) / 256);
  const int v = (variant >= 0 && variant < kNumEgaVariants) ? variant : kEgaDefault;
  const bool dig = ea.digest != nullptr;  // index digests (every variant has them)
  if (kEgaVariants[v].ray && ray_warps(ng) && ea.order) {
    jsc_ega_ray_launch(ea, v - kRayBase, dig, s);
    JSC_LAUNCH_CHECK();
    return JSC_OK;
  }
  if (kEgaVariants[v].lane) {
    const int lv = kEgaVariants[v].ray ? 4 : v - kLaneBase;
    if (ng <= 4) jsc_ega_lane_launch_s(ea, lv, dig, s);
    else jsc_ega_lane_launch_l(ea, lv, dig, s);
    JSC_LAUNCH_CHECK();
    return JSC_OK;
  }
  if (ng <= 2) jsc_ega_launch_g2(ea, g128, g256, v, dig, s);
  else if (ng <= 4) jsc_ega_launch_g4(ea, g128, g256, v, dig, s);
  else if (ng <= 8) jsc_ega_launch_g8(ea, g128, g256, v, dig, s);
  else jsc_ega_launch_gmax(ea, g128, g256, v, dig, s);
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

static void ev_record(jsc_batch *b, int k, int end, cudaStream_t s) {
  if (b->timing) cudaEventRecord(b->ev[2 * k + end], s);
  if (end) b->ran[k] = 1;
}

static void fill_ray_args(const jsc_batch *b, RayArgs &ra) {
  const jsc_model *m = b->m;
  const int nr = b->n_rays;
  memset(&ra, 0, sizeof(ra));
  ra.n_rays = nr;
  ra.ng = b->cfg.ng;
  ra.nw = b->cfg.nw;
  ra.ig_h2o = m->dv.ig_h2o;
  ra.n_levels = b->n_levels;
  ra.refrac = b->cfg.refrac;
  ra.rayds = b->cfg.rayds;
  ra.raydz = b->cfg.raydz;
  ra.ray_atm = b->d_ray_atm;
  ra.atm_off = b->d_atm_off;
  ra.time = b->d_ray;
  ra.obsz = b->d_ray + (size_t)nr;
  ra.obslon = b->d_ray + 2 * (size_t)nr;
  ra.obslat = b->d_ray + 3 * (size_t)nr;
  ra.vpz = b->d_ray + 4 * (size_t)nr;
  ra.vplon = b->d_ray + 5 * (size_t)nr;
  ra.vplat = b->d_ray + 6 * (size_t)nr;
  ra.z = b->d_z;
  ra.p = b->d_p;
  ra.t = b->d_t;
  ra.q = b->d_q;
  ra.k = b->d_k;
  ra.zmin = b->d_zmin;
  ra.zmax = b->d_zmax;
  ra.nlos = b->d_nlos;
  ra.los_off = b->d_los_off;
  ra.W = b->W;
  ra.tsurf = b->d_tsurf;
  ra.tp = b->d_tp;
  ra.status = b->d_status;
  ra.ip = b->ip;
  ra.n_prof = b->n_atm;
  ra.psurf = b->d_psurf;
  ra.lat = b->d_lat;
  ra.cz = b->cz;
  ra.cx = b->cx;
}

// Counting or storing ray-tracing pass with the batch's interpolation; the
// pencil batches of a fixed-capacity round pull their rays from the device
// queue with a persistent grid (7 blocks of 128 per SM, the kernel's cap).
template <bool STORE>
static int launch_raytrace(const jsc_batch *b, const RayArgs &ra, cudaStream_t s) {
  if (b->d_live) {
    JSC_CUDA_TRY(cudaMemsetAsync(b->d_qhead, 0, sizeof(unsigned), s));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->m->device);
    const unsigned g = (unsigned)(sms * 7);
    if (b->ip == 2) raytrace_queue_kernel<STORE, 2><<<g, 128, 0, s>>>(ra, b->d_qhead, b->d_live);
    else if (b->ip == 3) raytrace_queue_kernel<STORE, 3><<<g, 128, 0, s>>>(ra, b->d_qhead, b->d_live);
    else raytrace_queue_kernel<STORE><<<g, 128, 0, s>>>(ra, b->d_qhead, b->d_live);
    return JSC_OK;
  }
  const unsigned g = (unsigned)((ra.n_rays + 127) / 128);
  if (b->ip == 2) raytrace_kernel<STORE, 2><<<g, 128, 0, s>>>(ra);
  else if (b->ip == 3) raytrace_kernel<STORE, 3><<<g, 128, 0, s>>>(ra);
  else raytrace_kernel<STORE><<<g, 128, 0, s>>>(ra);
  return JSC_OK;
}

// Live rays of the pencil batches of round `first` (chunk points): the
// secondary pencils (nalpha per listed point) and the solar pencils.
static __global__ void round_live_kernel(const unsigned long long *n_listed, int64_t first,
                                         int chunk, int nalpha, int *live_sec, int *live_sun) {
  const int64_t left = (int64_t)*n_listed - first;
  const int pts = left <= 0 ? 0 : (left < chunk ? (int)left : chunk);
  *live_sec = pts * nalpha;
  *live_sun = pts;
}

static int batch_run(jsc_batch *b, cudaStream_t s);
static int run_hydro(jsc_batch *b, cudaStream_t s);

// Fixed-capacity runs: rays whose line of sight did not fit (the storing
// pass flagged them) keep only the points inside the buffer, so that no
// later kernel reads past it.
static __global__ void clamp_los_kernel(int *nlos, const int64_t *off, int n, int64_t cap) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int64_t room = cap - off[r];
  if (room < nlos[r]) nlos[r] = room > 0 ? (int)room : 0;
}

// OR a child batch's device status into its parent's.
static __global__ void status_or_kernel(unsigned *dst, const unsigned *src) { *dst |= *src; }

// A child batch for the secondary (depth - 1) or solar (depth 0) pencils
// of this batch's scattering points, with room for max_rays rays.
static int ensure_child(jsc_batch *b, jsc_batch **pc, int max_rays, int depth, int los_per_ray = 128) {
  jsc_batch *c = *pc;
  if (c && c->max_rays >= max_rays && c->max_seg >= (int64_t)max_rays * los_per_ray) {
    c->ega_variant = b->ega_variant;  // the parent's current launch variant
    return JSC_OK;
  }
  jsc_batch_destroy(c);
  *pc = nullptr;
  int st = jsc_batch_create(b->m, b->ctl, b->max_atm, b->max_levels, max_rays,
                            (int64_t)max_rays * los_per_ray, &c);
  if (st) return st;
  c->cfg.hydz = -1;  // profiles arrive hydrostatically balanced
  c->depth = depth;
  c->inner = 1;
  memcpy(c->nalpha_at, b->nalpha_at, sizeof(b->nalpha_at));
  c->nalpha = (depth <= JSC_MAX_DEPTH && b->nalpha_at[depth]) ? b->nalpha_at[depth] : b->nalpha;
  sca_alpha(c->alpha, c->nalpha);
  memcpy(c->sur_at, b->sur_at, sizeof(b->sur_at));
  memcpy(c->sur_tol_at, b->sur_tol_at, sizeof(b->sur_tol_at));
  memcpy(c->sur_stride_at, b->sur_stride_at, sizeof(b->sur_stride_at));
  if (depth >= 1 && depth <= JSC_MAX_DEPTH && c->sur_at[depth]) {
    c->sur = c->sur_at[depth];
    c->sur_on = 1;
    c->sur_tol = c->sur_tol_at[depth];
    c->sur_stride = c->sur_stride_at[depth];
  }
  c->ega_variant = b->ega_variant;
  if ((st = jsc_batch_set_aero(c, b->h_aero))) {
    jsc_batch_destroy(c);
    return st;
  }
  *pc = c;
  return JSC_OK;
}

// The child sees this batch's profiles, with the balanced pressures.
static int copy_profiles(const jsc_batch *b, jsc_batch *c, cudaStream_t s) {
  const size_t nl = (size_t)b->n_levels;
  c->n_atm = b->n_atm;
  c->n_levels = b->n_levels;
#define D2D(dst, src, n) \
  JSC_CUDA_TRY(cudaMemcpyAsync((dst), (src), (n) * sizeof(*(src)), cudaMemcpyDeviceToDevice, s))
  D2D(c->d_atm_off, b->d_atm_off, (size_t)b->n_atm + 1);
  D2D(c->d_z, b->d_z, nl);
  D2D(c->d_lon, b->d_lon, nl);
  D2D(c->d_lat, b->d_lat, nl);
  D2D(c->d_p_in, b->d_p, nl);
  D2D(c->d_t, b->d_t, nl);
  if (b->cfg.ng > 0) D2D(c->d_q, b->d_q, nl * b->cfg.ng);
  if (b->cfg.nw > 0) D2D(c->d_k, b->d_k, nl * b->cfg.nw);
#undef D2D
  return JSC_OK;
}

// Room for n scattering point records, their profiles and sources.
static int reserve_points(jsc_batch *b, int64_t n_sp) {
  if (n_sp <= b->max_sp) return JSC_OK;
  int st;
  cudaFree(b->d_sp);
  cudaFree(b->d_sp_atm);
  cudaFree(b->d_src);
  b->d_sp = b->d_src = nullptr;
  b->d_sp_atm = nullptr;
  b->max_sp = 0;
  const int64_t n = n_sp + n_sp / 4 + 256;
  if ((st = jsc_dmalloc(&b->d_sp, (size_t)n * JSC_SP_REC))) return st;
  if ((st = jsc_dmalloc(&b->d_sp_atm, (size_t)n))) return st;
  if ((st = jsc_dmalloc(&b->d_src, (size_t)n * b->cfg.nd))) return st;
  b->max_sp = n;
  return JSC_OK;
}

// Scattering points per ray and their list (src/forwardmodel.c:317-331).
static int list_scattering_points(jsc_batch *b, cudaStream_t s) {
  const int nr = b->n_rays;
  int st;
  if (!b->d_nsp) {
    if ((st = jsc_dmalloc(&b->d_nsp, (size_t)b->max_rays))) return st;
    if ((st = jsc_dmalloc(&b->d_sp_off, (size_t)b->max_rays + 1))) return st;
  }
  SpArgs sa;
  sa.n_rays = nr;
  sa.W = b->W;
  sa.nlos = b->d_nlos;
  sa.los_off = b->d_los_off;
  sa.geo = b->d_geo;
  sa.pts = b->d_pts;
  sa.time = b->d_ray;
  sa.ray_atm = b->d_ray_atm;
  sa.nsp = b->d_nsp;
  sa.sp_off = b->d_sp_off;
  sa.sp = nullptr;
  sa.sp_atm = nullptr;
  sa.max_sp = 0;
  sa.nlos_mut = nullptr;
  sa.status = b->d_status;
  sa.n_listed = nullptr;
  sp_count_kernel<<<(nr + 127) / 128, 128, 0, s>>>(sa);
  JSC_LAUNCH_CHECK();
  if ((st = launch_scan(b, b->d_nsp, nr, b->d_sp_off, s))) return st;
  JSC_CUDA_TRY(cudaMemcpyAsync(b->h_total, b->d_sp_off + nr, sizeof(int64_t),
                               cudaMemcpyDeviceToHost, s));
  JSC_CUDA_TRY(cudaStreamSynchronize(s));
  b->n_sp = *b->h_total;
  if ((st = reserve_points(b, b->n_sp))) return st;
  if (b->n_sp == 0) return JSC_OK;
  sa.sp = b->d_sp;
  sa.sp_atm = b->d_sp_atm;
  sp_list_kernel<<<(nr + 127) / 128, 128, 0, s>>>(sa);
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

// Scattering points per chunk: the secondary pencils of a chunk run as one
// child batch of chunk * nalpha rays.
// Scattering points per child-batch round of the 1-D source: large rounds
// keep the GPU busy between the host's LOS-size reads, bounded so the
// child's per-(LOS point, channel) buffers stay near 20 GB (32768 points at
// 16 channels, 8192 at 64).
static int64_t scatter_chunk(int nd) {
  const int64_t c = 524288 / (nd > 0 ? nd : 1);
  return c < 8192 ? 8192 : (c > 32768 ? 32768 : c);
}

// Scattering source of every scattering point (srcfunc_sca,
// src/scatter.c:643-662): thermal radiation from the secondary pencils,
// then the solar term.
// The plain scattering source (srcfunc_sca) of n point records sp
// (profiles sp_atm) into src [n][nd].
// Solar term of n scattering points (srcfunc_sca_sun, src/scatter.c:899-995):
// the refracted sun direction by repeated ray tracing, the solar pencils as
// a child batch, and the phase-function weighted solar source added to src.
static int sun_sources(jsc_batch *b, const double *sp, const int *sp_atm, int n, double *src,
                       cudaStream_t s, const int64_t *n_total = nullptr, int64_t first = 0) {
  jsc_batch *sc = b->sun_child;
  SunArgs sn;
  fill_ray_args(b, sn.ra);
  sn.n_pts = n;
  sn.n_total = n_total;
  sn.first = first;
  sn.sp = sp;
  sn.sp_atm = sp_atm;
  sn.n_alti = b->n_alti;
  sn.altimax = b->altimax;
  sn.altimin = b->altimin;
  sn.alti = b->d_aero + 3 * NLMAX;
  sn.ray_atm = sc->d_ray_atm;
  sn.ray = sc->d_ray;
  sn.theta2 = b->d_theta2;
  sc->n_rays = n;
  if (b->ip != 1) {  // surface positions for the direction search
    const int np = b->ip == 2 ? b->n_atm : b->n_levels;
    psurf_kernel<<<(np + 127) / 128, 128, 0, s>>>(np, b->ip == 3, b->d_atm_off, b->d_lon,
                                                  b->d_lat, b->d_psurf);
    JSC_LAUNCH_CHECK();
  }
  if (b->ip == 2) sun_kernel<2><<<(n + 127) / 128, 128, 0, s>>>(sn);
  else if (b->ip == 3) sun_kernel<3><<<(n + 127) / 128, 128, 0, s>>>(sn);
  else sun_kernel<<<(n + 127) / 128, 128, 0, s>>>(sn);
  JSC_LAUNCH_CHECK();
  int st = batch_run(sc, s);
  if (st) return st;
  status_or_kernel<<<1, 1, 0, s>>>(b->d_status, sc->d_status);
  JSC_LAUNCH_CHECK();
  SunAddArgs aa;
  aa.n_pts = n;
  aa.nd = b->cfg.nd;
  aa.sp = sp;
  aa.theta2 = b->d_theta2;
  aa.tau = sc->d_tau;
  aa.phase = b->d_phase;
  aa.planck_sun = b->d_planck_sun;
  aa.src = src;
  sun_add_kernel<<<(n * b->cfg.nd + 127) / 128, 128, 0, s>>>(aa);
  JSC_LAUNCH_CHECK();
  return JSC_OK;
}

// Scattering points per chunk of the 3-D source (32,400 pencils each).
static const int64_t kScatterChunk3 = 16;

static int plain_sources(jsc_batch *b, const double *sp, const int *sp_atm, int64_t n_pts,
                         double *src, cudaStream_t s) {
  int st = JSC_OK;
  if (n_pts <= 0) return JSC_OK;
  const int nd = b->cfg.nd, na = b->nalpha;
  const bool three_d = b->ip != 1;  // srcfunc_sca_3d (src/scatter.c:654-657)
  const int64_t cap = three_d ? kScatterChunk3 : scatter_chunk(nd);
  const int64_t chunk = n_pts < cap ? n_pts : cap;
  const int64_t per_pt = three_d ? JSC_NDIR3 : na;
  if ((st = ensure_child(b, &b->child, (int)(chunk * per_pt), b->depth - 1))) return st;
  if ((st = ensure_child(b, &b->sun_child, (int)chunk, 0))) return st;
  if (!b->d_planck_sun) {
    double h[NDMAX];
    for (int id = 0; id < nd; id++) h[id] = planck(JSC_TSUN, b->m->nu[id]);
    if ((st = jsc_dmalloc(&b->d_planck_sun, (size_t)nd))) return st;
    JSC_CUDA_TRY(cudaMemcpy(b->d_planck_sun, h, (size_t)nd * sizeof(double),
                            cudaMemcpyHostToDevice));
  }
  if (b->n_theta2 < b->sun_child->max_rays) {
    cudaFree(b->d_theta2);
    b->d_theta2 = nullptr;
    b->n_theta2 = 0;
    if ((st = jsc_dmalloc(&b->d_theta2, (size_t)b->sun_child->max_rays))) return st;
    b->n_theta2 = b->sun_child->max_rays;
  }
  if ((st = copy_profiles(b, b->child, s))) return st;
  if ((st = copy_profiles(b, b->sun_child, s))) return st;

  jsc_batch *c = b->child, *sc = b->sun_child;
  const size_t shmem = ((size_t)JSC_NTH_SCA * nd + (size_t)na * (nd | 1) + 4 * JSC_NTH_SCA +
                        (JSC_INT_THREADS / 32) * JSC_INT_CH + (size_t)na * (JSC_INT_CH + 1) +
                        (size_t)na) *
                       sizeof(double);
  if (shmem > 48 * 1024)
    JSC_CUDA_TRY(cudaFuncSetAttribute(sp_integral_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  for (int64_t c0 = 0; c0 < n_pts && three_d; c0 += chunk) {
    const int n = (int)((n_pts - c0) < chunk ? (n_pts - c0) : chunk);
    // Pencils in every direction around the line of sight (src/scatter.c:835-856).
    Spawn3Args pa;
    pa.n_pts = n;
    pa.sp = sp + c0 * JSC_SP_REC;
    pa.sp_atm = sp_atm + c0;
    pa.ray_atm = c->d_ray_atm;
    pa.ray = c->d_ray;
    c->n_rays = (int)(n * JSC_NDIR3);
    sp_spawn3_kernel<<<(unsigned)(((int64_t)n * JSC_NDIR3 + 127) / 128), 128, 0, s>>>(pa);
    JSC_LAUNCH_CHECK();
    if ((st = batch_run(c, s))) return st;
    status_or_kernel<<<1, 1, 0, s>>>(b->d_status, c->d_status);
    JSC_LAUNCH_CHECK();
    Integral3Args ia;
    ia.n_pts = n;
    ia.nd = nd;
    ia.sp = pa.sp;
    ia.rad = c->d_rad;
    ia.phase = b->d_phase;
    ia.src = src + c0 * nd;
    sp_integral3_kernel<<<n, JSC_INT_THREADS, 0, s>>>(ia);
    JSC_LAUNCH_CHECK();
    if ((st = sun_sources(b, pa.sp, pa.sp_atm, n, src + c0 * nd, s))) return st;
  }
  for (int64_t c0 = 0; c0 < n_pts && !three_d; c0 += chunk) {
    const int n = (int)((n_pts - c0) < chunk ? (n_pts - c0) : chunk);
    // Secondary pencils (src/scatter.c:717-736).
    SpawnArgs pa;
    pa.n_pts = n;
    pa.nalpha = na;
    pa.n_total = nullptr;
    pa.first = c0;
    pa.sp = sp + c0 * JSC_SP_REC;
    pa.sp_atm = sp_atm + c0;
    memcpy(pa.alpha, b->alpha, sizeof(pa.alpha));
    pa.ray_atm = c->d_ray_atm;
    pa.ray = c->d_ray;
    c->n_rays = n * na;
    sp_spawn_kernel<<<(n * na + 127) / 128, 128, 0, s>>>(pa);
    JSC_LAUNCH_CHECK();
    if ((st = batch_run(c, s))) return st;
    status_or_kernel<<<1, 1, 0, s>>>(b->d_status, c->d_status);
    JSC_LAUNCH_CHECK();
    // Source integral over the sphere (src/scatter.c:737-805).
    IntegralArgs ia;
    ia.n_pts = n;
    ia.nalpha = na;
    ia.n_total = nullptr;
    ia.first = c0;
    ia.nd = nd;
    ia.nl = b->aero_nl;
    ia.sp = pa.sp;
    memcpy(ia.alpha, b->alpha, sizeof(ia.alpha));
    ia.rad = c->d_rad;
    ia.phase = b->d_phase;
    ia.src = src + c0 * nd;
    sp_integral_kernel<<<n, JSC_INT_THREADS, shmem, s>>>(ia);
    JSC_LAUNCH_CHECK();
    if ((st = sun_sources(b, pa.sp, pa.sp_atm, n, src + c0 * nd, s))) return st;
  }
  return JSC_OK;
}

// Scattering sources of a fixed-capacity run (single scattering, IP 1),
// without a host read-back: the point list is counted and placed on the
// device (with its total in d_sp_off[n_rays]), then fx_rounds rounds of
// fx_chunk points each spawn their secondary pencils into the child batch
// (null pencils past the device count), run it, integrate the sources and
// add the solar term.  The launch sequence is the same for every input, so
// the run can be captured into a CUDA graph.  Points beyond the capacity
// fx_max_sp empty their ray's LOS and set JSC_DEV_ERR_QUEUE.
static int fixed_sources(jsc_batch *b, cudaStream_t s) {
  const int nr = b->n_rays, nd = b->cfg.nd, na = b->nalpha;
  int st;
  SpArgs sa;
  sa.n_rays = nr;
  sa.W = b->W;
  sa.nlos = b->d_nlos;
  sa.los_off = b->d_los_off;
  sa.geo = b->d_geo;
  sa.pts = b->d_pts;
  sa.time = b->d_ray;
  sa.ray_atm = b->d_ray_atm;
  sa.nsp = b->d_nsp;
  sa.sp_off = b->d_sp_off;
  sa.sp = b->d_sp;
  sa.sp_atm = b->d_sp_atm;
  sa.max_sp = b->fx_max_sp;
  sa.nlos_mut = b->d_nlos;
  sa.status = b->d_status;
  sa.n_listed = b->d_sp_listed;
  sp_count_kernel<<<(nr + 127) / 128, 128, 0, s>>>(sa);
  JSC_LAUNCH_CHECK();
  if ((st = launch_scan(b, b->d_nsp, nr, b->d_sp_off, s))) return st;
  sp_listed_init_kernel<<<1, 1, 0, s>>>(b->d_sp_off + nr, b->fx_max_sp, b->d_sp_listed);
  JSC_LAUNCH_CHECK();
  sp_list_kernel<<<(nr + 127) / 128, 128, 0, s>>>(sa);
  JSC_LAUNCH_CHECK();
  if ((st = copy_profiles(b, b->child, s))) return st;
  if ((st = copy_profiles(b, b->sun_child, s))) return st;
  const int64_t *n_total = reinterpret_cast<const int64_t *>(b->d_sp_listed);
  const int chunk = (int)b->fx_chunk;
  jsc_batch *c = b->child;
  const size_t shmem = ((size_t)JSC_NTH_SCA * nd + (size_t)na * (nd | 1) + 4 * JSC_NTH_SCA +
                        (JSC_INT_THREADS / 32) * JSC_INT_CH + (size_t)na * (JSC_INT_CH + 1) +
                        (size_t)na) *
                       sizeof(double);
  for (int r = 0; r < b->fx_rounds; r++) {
    const int64_t c0 = (int64_t)r * chunk;
    SpawnArgs pa;
    pa.n_pts = chunk;
    pa.nalpha = na;
    pa.n_total = n_total;
    pa.first = c0;
    pa.sp = b->d_sp + c0 * JSC_SP_REC;
    pa.sp_atm = b->d_sp_atm + c0;
    memcpy(pa.alpha, b->alpha, sizeof(pa.alpha));
    pa.ray_atm = c->d_ray_atm;
    pa.ray = c->d_ray;
    c->n_rays = chunk * na;
    sp_spawn_kernel<<<(chunk * na + 127) / 128, 128, 0, s>>>(pa);
    JSC_LAUNCH_CHECK();
    round_live_kernel<<<1, 1, 0, s>>>(b->d_sp_listed, c0, chunk, na, c->d_live,
                                      b->sun_child->d_live);
    JSC_LAUNCH_CHECK();
    if ((st = batch_run(c, s))) return st;
    status_or_kernel<<<1, 1, 0, s>>>(b->d_status, c->d_status);
    JSC_LAUNCH_CHECK();
    IntegralArgs ia;
    ia.n_pts = chunk;
    ia.nalpha = na;
    ia.n_total = n_total;
    ia.first = c0;
    ia.nd = nd;
    ia.nl = b->aero_nl;
    ia.sp = pa.sp;
    memcpy(ia.alpha, b->alpha, sizeof(ia.alpha));
    ia.rad = c->d_rad;
    ia.phase = b->d_phase;
    ia.src = b->d_src + c0 * nd;
    sp_integral_kernel<<<chunk, JSC_INT_THREADS, shmem, s>>>(ia);
    JSC_LAUNCH_CHECK();
    if ((st = sun_sources(b, pa.sp, pa.sp_atm, chunk, b->d_src + c0 * nd, s, n_total, c0)))
      return st;
  }
  return JSC_OK;
}

// Everything a fixed-capacity single-scattering run uses, allocated before
// the first run (a captured run cannot allocate): the point list of
// fx_max_sp points, the child batches of one round (fx_chunk points: their
// secondary and solar pencils, themselves fixed-capacity), the solar data.
static int prepare_fixed_scattering(jsc_batch *b) {
  if (b->depth != 1 || b->ip != 1 || b->sur_on) {
    jsc_set_error(JSC_ERR_UNSUPPORTED, "fixed-capacity scattering runs cover single scattering "
                                       "(SCA_MULT=1) in 1-D atmospheres without a surrogate");
    return JSC_ERR_UNSUPPORTED;
  }
  if (!b->h_aero || !b->d_aero) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_fixed with scattering: call jsc_batch_set_aero first");
    return JSC_ERR_ARG;
  }
  const int nd = b->cfg.nd, na = b->nalpha;
  int st;
  int64_t chunk = scatter_chunk(nd);
  const int64_t want = b->fx_points_req > 0 ? b->fx_points_req
                                            : (int64_t)b->max_rays * JSC_FIXED_POINTS_PER_RAY;
  if (chunk > want) chunk = want;
  b->fx_chunk = chunk;
  b->fx_rounds = (int)((want + chunk - 1) / chunk);
  b->fx_max_sp = (int64_t)b->fx_rounds * chunk;
  if (!b->d_nsp) {
    if ((st = jsc_dmalloc(&b->d_nsp, (size_t)b->max_rays))) return st;
    if ((st = jsc_dmalloc(&b->d_sp_off, (size_t)b->max_rays + 1))) return st;
  }
  if ((st = reserve_points(b, b->fx_max_sp))) return st;
  if (!b->d_sp_listed && (st = jsc_dmalloc(&b->d_sp_listed, 1))) return st;
  if ((st = ensure_child(b, &b->child, (int)(chunk * na), 0, JSC_FIXED_PENCIL_LOS))) return st;
  if ((st = ensure_child(b, &b->sun_child, (int)chunk, 0, JSC_FIXED_SUN_LOS))) return st;
  if ((st = jsc_batch_set_fixed(b->child, 1))) return st;
  if ((st = jsc_batch_set_fixed(b->sun_child, 1))) return st;
  for (jsc_batch *c : {b->child, b->sun_child}) {
    if (!c->d_live && (st = jsc_dmalloc(&c->d_live, 1))) return st;
    if (!c->d_qhead && (st = jsc_dmalloc(&c->d_qhead, 1))) return st;
  }
  if (!b->d_planck_sun) {
    double h[NDMAX];
    for (int id = 0; id < nd; id++) h[id] = planck(JSC_TSUN, b->m->nu[id]);
    if ((st = jsc_dmalloc(&b->d_planck_sun, (size_t)nd))) return st;
    JSC_CUDA_TRY(cudaMemcpy(b->d_planck_sun, h, (size_t)nd * sizeof(double),
                            cudaMemcpyHostToDevice));
  }
  if (b->n_theta2 < b->sun_child->max_rays) {
    cudaFree(b->d_theta2);
    b->d_theta2 = nullptr;
    b->n_theta2 = 0;
    if ((st = jsc_dmalloc(&b->d_theta2, (size_t)b->sun_child->max_rays))) return st;
    b->n_theta2 = b->sun_child->max_rays;
  }
  const size_t shmem = ((size_t)JSC_NTH_SCA * nd + (size_t)na * (nd | 1) + 4 * JSC_NTH_SCA +
                        (JSC_INT_THREADS / 32) * JSC_INT_CH + (size_t)na * (JSC_INT_CH + 1) +
                        (size_t)na) *
                       sizeof(double);
  if (shmem > 48 * 1024)
    JSC_CUDA_TRY(cudaFuncSetAttribute(sp_integral_kernel,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shmem));
  return JSC_OK;
}

extern "C" int jsc_batch_set_fixed_points(jsc_batch *b, int64_t max_points) {
  if (!b || max_points < 0) return JSC_ERR_ARG;
  b->fx_points_req = max_points;
  return JSC_OK;
}

// Marks of the surrogate pass: 0 surrogate only, 1 outside the envelope
// (plain), 2 inside and sampled for the accuracy check (both).
static __global__ void sur_mark_kernel(int n, const float *feat, SurEnvelope env, int stride,
                                       int *mark) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  bool in = true;
  for (int c = 0; c < SUR_NF; c++) {
    const float v = feat[(size_t)k * SUR_NF + c];
    if (!(v >= env.lo[c] && v <= env.hi[c])) in = false;
  }
  mark[k] = !in ? 1 : ((stride > 0 && k % stride == 0) ? 2 : 0);
}

// Compact the marked points: idx[] of marks != 0 in order (one block).
static __global__ void sur_compact_kernel(int n, const int *mark, int *idx, int *count) {
  __shared__ int base;
  if (threadIdx.x == 0) base = 0;
  __syncthreads();
  for (int k0 = 0; k0 < n; k0 += blockDim.x) {
    const int k = k0 + threadIdx.x;
    const int f = (k < n && mark[k] != 0) ? 1 : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    __shared__ int wsum[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wsum[w] = __popc(bal);
    __syncthreads();
    int off = 0;
    for (int i = 0; i < w; i++) off += wsum[i];
    if (f) idx[base + off + __popc(bal & ((1u << lane) - 1))] = k;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int i = 0; i < (int)(blockDim.x >> 5); i++) tot += wsum[i];
      base += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *count = base;
}

static __global__ void sur_gather_kernel(int m, const int *idx, const double *sp, const int *sp_atm,
                                         double *sp_sub, int *atm_sub) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int k = idx[i];
  for (int c = 0; c < JSC_SP_REC; c++) sp_sub[(size_t)i * JSC_SP_REC + c] = sp[(size_t)k * JSC_SP_REC + c];
  atm_sub[i] = sp_atm[k];
}

// Fallback points take the plain source; checked points compare the
// surrogate's source with it.  The source enters the radiance through the
// segment source ((bext - af bs) B + af bs S) / bext
// (src/forwardmodel.c:344-349), where af bs / bext <= bs / be, the layer's
// single-scattering albedo; the check measures omega |dS| / S, which bounds
// the relative error of the segment source: its largest value (as float
// bits) and its sum over the checked (point, channel) pairs.
static __global__ void sur_merge_kernel(int m, int nd, const int *idx, const int *mark,
                                        const double *sp, const double *beta, int nl,
                                        const double *src_sub, double *src, unsigned *maxerr,
                                        float *errsum) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  float e = 0.0f;
  if (t < m * nd) {
    const int i = t / nd, d = t - i * nd, k = idx[i];
    const double plain = src_sub[(size_t)i * nd + d];
    double *dst = src + (size_t)k * nd + d;
    if (mark[k] == 1) {
      *dst = plain;
    } else {
      const int il = (int)sp[(size_t)k * JSC_SP_REC + SP_IL];
      const double be = beta[(size_t)il * nd + d], bs = beta[(size_t)(nl + il) * nd + d];
      const double omega = be > 0 ? fmin(fmax(bs / be, 0.0), 1.0) : 1.0;
      e = (float)(omega * fabs(*dst - plain) / fmax(fabs(plain), 1e-300));
      e = e == e ? e : 3.0e38f;
      atomicMax(maxerr, __float_as_uint(e));
    }
  }
  // every thread of the block takes part (blockDim.x is a multiple of 32)
  for (int off = 16; off > 0; off >>= 1) e += __shfl_down_sync(0xffffffffu, e, off);
  if ((threadIdx.x & 31) == 0 && e > 0.0f) atomicAdd(errsum, e);
}

// Scattering source of every scattering point (srcfunc_sca,
// src/scatter.c:643-662): the plain path (secondary and solar pencils), or,
// with a trained surrogate attached, the surrogate for points inside its
// envelope and the plain path for the rest and for a sample of the inside
// points, which checks the surrogate; if a checked point deviates by more
// than the tolerance the whole batch takes the plain path.
static int fixed_sources(jsc_batch *b, cudaStream_t s);

// Fallback (outside the envelope) and checked points of the last marking.
static int count_marks(jsc_batch *b, int n) {
  int *hm = (int *)malloc((size_t)n * sizeof(int));
  if (!hm) return JSC_ERR_NOMEM;
  if (cudaMemcpy(hm, b->d_mark, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    free(hm);
    jsc_set_error(JSC_ERR_CUDA, "surrogate marks read-back");
    return JSC_ERR_CUDA;
  }
  for (int k = 0; k < n; k++) {
    if (hm[k] == 1) b->sur_fallback++;
    else if (hm[k] == 2) b->sur_checked++;
  }
  free(hm);
  return JSC_OK;
}

// Zero the surrogate statistics of b and its children.
static void sur_stats_reset(jsc_batch *b) {
  for (jsc_batch *c = b; c; c = c->child) {
    c->sur_points = c->sur_fallback = c->sur_checked = 0;
    c->sur_maxerr = 0;
    c->sur_errsum = 0;
    c->sur_errn = 0;
    c->sur_runs = c->sur_used_runs = 0;
  }
}

static int scatter_sources(jsc_batch *b, cudaStream_t s) {
  if (b->fixed) return fixed_sources(b, s);
  int st = list_scattering_points(b, s);
  if (st || b->n_sp == 0) return st;
  const int nd = b->cfg.nd;
  const int n = (int)b->n_sp;
  // statistics add up over the chunks of one jsc_batch_run (a child batch
  // runs once per chunk of its parent)
  b->sur_points += b->n_sp;
  b->sur_runs++;
  if (!(b->sur && b->sur_on && jsc_sur_trained(b->sur) && jsc_sur_nout(b->sur) == nd))
    return plain_sources(b, b->d_sp, b->d_sp_atm, b->n_sp, b->d_src, s);
  if (b->sur_cap < b->n_sp) {
    cudaFree(b->d_feat);
    cudaFree(b->d_mark);
    cudaFree(b->d_idx);
    cudaFree(b->d_sp_sub);
    cudaFree(b->d_atm_sub);
    cudaFree(b->d_src_sub);
    b->d_feat = nullptr;
    b->d_mark = b->d_idx = b->d_atm_sub = nullptr;
    b->d_sp_sub = b->d_src_sub = nullptr;
    b->sur_cap = 0;
    const int64_t cap = b->max_sp;
    if ((st = jsc_dmalloc(&b->d_feat, (size_t)cap * SUR_NF))) return st;
    if ((st = jsc_dmalloc(&b->d_mark, (size_t)cap))) return st;
    if ((st = jsc_dmalloc(&b->d_idx, (size_t)cap + 2))) return st;  // + count, error sum
    if ((st = jsc_dmalloc(&b->d_sp_sub, (size_t)cap * JSC_SP_REC))) return st;
    if ((st = jsc_dmalloc(&b->d_atm_sub, (size_t)cap))) return st;
    if ((st = jsc_dmalloc(&b->d_src_sub, (size_t)cap * nd))) return st;
    b->sur_cap = cap;
  }
  if ((st = jsc_sur_features(n, b->d_sp, b->d_feat, s))) return st;
  SurEnvelope env;
  jsc_sur_envelope(b->sur, env.lo, env.hi);
  sur_mark_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, b->d_feat, env, b->sur_stride, b->d_mark);
  JSC_LAUNCH_CHECK();
  ev_record(b, JSC_T_SUR, 0, s);
  if ((st = jsc_sur_infer(b->sur, n, b->d_feat, b->d_src, nd, s))) return st;
  ev_record(b, JSC_T_SUR, 1, s);
  sur_compact_kernel<<<1, 1024, 0, s>>>(n, b->d_mark, b->d_idx, b->d_idx + b->sur_cap);
  JSC_LAUNCH_CHECK();
  int m = 0;
  JSC_CUDA_TRY(cudaMemcpyAsync(b->h_total, b->d_idx + b->sur_cap, sizeof(int),
                               cudaMemcpyDeviceToHost, s));
  JSC_CUDA_TRY(cudaStreamSynchronize(s));
  m = *(int *)b->h_total;
  if (m > 0) {
    sur_gather_kernel<<<(m + 127) / 128, 128, 0, s>>>(m, b->d_idx, b->d_sp, b->d_sp_atm,
                                                      b->d_sp_sub, b->d_atm_sub);
    JSC_LAUNCH_CHECK();
    if ((st = plain_sources(b, b->d_sp_sub, b->d_atm_sub, m, b->d_src_sub, s))) return st;
    // the count word becomes the largest error, the word after it the sum
    unsigned *d_err = (unsigned *)b->d_idx + b->sur_cap;
    JSC_CUDA_TRY(cudaMemsetAsync(d_err, 0, 2 * sizeof(unsigned), s));
    sur_merge_kernel<<<(m * nd + 127) / 128, 128, 0, s>>>(m, nd, b->d_idx, b->d_mark, b->d_sp,
                                                          b->d_beta, b->aero_nl, b->d_src_sub,
                                                          b->d_src, d_err, (float *)(d_err + 1));
    JSC_LAUNCH_CHECK();
    JSC_CUDA_TRY(cudaMemcpyAsync(b->h_total, d_err, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost,
                                 s));
    JSC_CUDA_TRY(cudaStreamSynchronize(s));
    float e, sum;
    memcpy(&e, (const unsigned char *)b->h_total, sizeof(e));
    memcpy(&sum, (const unsigned char *)b->h_total + sizeof(float), sizeof(sum));
    const int64_t before = b->sur_checked;
    if ((st = count_marks(b, n))) return st;
    const int64_t pairs = (b->sur_checked - before) * nd;
    b->sur_maxerr = fmaxf(b->sur_maxerr, e);
    b->sur_errsum += sum;
    b->sur_errn += pairs;
    // The points of a scattering order below the top reach the radiance
    // only through the source integrals of the order above (each a sum
    // over pencils of line-of-sight integrals over many such points), so
    // their check bounds the mean deviation; the top order's sources enter
    // the radiance point by point, so its check bounds the largest one.
    const double crit = b->inner ? (pairs > 0 ? sum / (double)pairs : 0.0) : e;
    if (!(crit <= b->sur_tol)) {
      // the check missed the tolerance: this chunk takes the plain path
      b->sur_rejected++;
      return plain_sources(b, b->d_sp, b->d_sp_atm, b->n_sp, b->d_src, s);
    }
  } else if ((st = count_marks(b, n))) {
    return st;
  }
  b->sur_used_runs++;
  return JSC_OK;
}

extern "C" int jsc_batch_scatter_points(jsc_batch *b, int n, const double *x, const double *dx,
                                        const int *layer, const double *time, const int *prof,
                                        double *src, void *stream) {
  if (!b || n < 0 || (n > 0 && (!x || !dx || !layer || !time || !src))) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_scatter_points: invalid arguments");
    return JSC_ERR_ARG;
  }
  if (b->depth < 1 || !b->d_aero || b->n_atm < 1) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_scatter_points: needs a batch with SCA_N > 0, "
                               "SCA_MULT >= 1, jsc_batch_set_aero and uploaded profiles");
    return JSC_ERR_ARG;
  }
  for (int k = 0; k < n; k++)
    if (layer[k] < 0 || layer[k] >= b->aero_nl || (prof && (prof[k] < 0 || prof[k] >= b->n_atm))) {
      jsc_set_error(JSC_ERR_ARG, "jsc_batch_scatter_points: point %d names layer %d of %d or "
                    "profile %d of %d", k, layer[k], b->aero_nl, prof ? prof[k] : 0, b->n_atm);
      return JSC_ERR_ARG;
    }
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  (void)cudaGetLastError();
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return JSC_OK;
  int st = reserve_points(b, n);
  if (st) return st;
  double *rec = (double *)malloc((size_t)n * JSC_SP_REC * sizeof(double));
  int *pa = (int *)malloc((size_t)n * sizeof(int));
  if (!rec || !pa) {
    free(rec);
    free(pa);
    return JSC_ERR_NOMEM;
  }
  for (int k = 0; k < n; k++) {
    double *o = rec + (size_t)k * JSC_SP_REC;
    for (int i = 0; i < 3; i++) {
      o[SP_X + i] = x[3 * k + i];
      o[SP_DX + i] = dx[3 * k + i];
    }
    o[SP_IL] = layer[k];
    o[SP_TIME] = time[k];
    o[SP_P] = o[SP_T] = 0;  // read by the surrogate's features only
    pa[k] = prof ? prof[k] : 0;
  }
  for (int k = 0; k < JSC_T_N; k++) b->ran[k] = 0;
  cudaError_t e = cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_sp, rec, (size_t)n * JSC_SP_REC * sizeof(double),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->d_sp_atm, pa, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // rec and pa are freed next
  free(rec);
  free(pa);
  if (e != cudaSuccess) {
    jsc_set_error(JSC_ERR_CUDA, "jsc_batch_scatter_points: %s", cudaGetErrorString(e));
    return JSC_ERR_CUDA;
  }
  b->n_sp = n;
  if ((st = run_hydro(b, s))) return st;
  if ((st = plain_sources(b, b->d_sp, b->d_sp_atm, n, b->d_src, s))) return st;
  unsigned status = 0;
  JSC_CUDA_TRY(cudaMemcpyAsync(src, b->d_src, (size_t)n * b->cfg.nd * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
  JSC_CUDA_TRY(cudaMemcpyAsync(&status, b->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  JSC_CUDA_TRY(cudaStreamSynchronize(s));
  return map_status(status);
}

extern "C" int jsc_batch_run(jsc_batch *b, void *stream) {
  if (!b) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  (void)cudaGetLastError();  // launch checks below report this run's errors only
  sur_stats_reset(b);
  return batch_run(b, (cudaStream_t)stream);
}

// Hydrostatic balance of the uploaded profiles (when hydz >= 0) into d_p,
// and each profile's altitude range.
static int run_hydro(jsc_batch *b, cudaStream_t s) {
  const jsc_model *m = b->m;
  AtmArgs aa;
  aa.n_atm = b->n_atm;
  aa.n_levels = b->n_levels;
  aa.ng = b->cfg.ng;
  aa.nw = b->cfg.nw;
  aa.ig_h2o = m->dv.ig_h2o;
  aa.off = b->d_atm_off;
  aa.z = b->d_z;
  aa.lon = b->d_lon;
  aa.lat = b->d_lat;
  aa.p_in = b->d_p_in;
  aa.t = b->d_t;
  aa.q = b->d_q;
  aa.k = b->d_k;
  aa.p = b->d_p;
  aa.zmin = b->d_zmin;
  aa.zmax = b->d_zmax;
  aa.hydz = b->cfg.hydz;
  ev_record(b, JSC_T_HYDRO, 0, s);
  hydro_kernel<<<(b->n_atm + 127) / 128, 128, 0, s>>>(aa);
  JSC_LAUNCH_CHECK();
  ev_record(b, JSC_T_HYDRO, 1, s);
  return JSC_OK;
}

static int batch_run(jsc_batch *b, cudaStream_t s) {
  const jsc_model *m = b->m;
  const int nr = b->n_rays;
  for (int k = 0; k < JSC_T_N; k++) b->ran[k] = 0;
  JSC_CUDA_TRY(cudaMemsetAsync(b->d_status, 0, sizeof(unsigned), s));
  JSC_CUDA_TRY(cudaMemsetAsync(b->d_counters, 0, 2 * sizeof(unsigned long long), s));
  {
    int st = run_hydro(b, s);
    if (st) return st;
  }
  if (nr == 0) return JSC_OK;

  RayArgs ra;
  fill_ray_args(b, ra);
  if (m->n_grid == 1) {
    ra.grid_np = m->grid_np0;
    ra.grid_p = m->d_grid_p;
    ra.grid_nt = m->d_grid_nt;
    ra.grid_t = m->d_grid_t;
  }
  const bool refine = b->cfg.sca_n > 0;
  if (refine && !b->d_aero) {
    jsc_set_error(JSC_ERR_ARG, "SCA_N > 0 needs jsc_batch_set_aero before jsc_batch_run");
    return JSC_ERR_ARG;
  }
  ra.raw_q = refine;
  ra.nlos = refine ? b->d_nlos_b : b->d_nlos;
  ra.los_off = refine ? b->d_los_off_b : b->d_los_off;
  ev_record(b, JSC_T_RAYTRACE, 0, s);
  if (b->ip != 1) {  // surface positions of the profiles (IP 2) or levels (IP 3)
    const int n = b->ip == 2 ? b->n_atm : b->n_levels;
    psurf_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, b->ip == 3, b->d_atm_off, b->d_lon, b->d_lat,
                                                 b->d_psurf);
    JSC_LAUNCH_CHECK();
  }
  if (b->d_live) {  // rays the queue leaves alone keep no LOS and no surface
    JSC_CUDA_TRY(cudaMemsetAsync(ra.nlos, 0, (size_t)nr * sizeof(int), s));
    JSC_CUDA_TRY(cudaMemsetAsync(b->d_tsurf, 0, (size_t)nr * sizeof(double), s));
  }
  {
    const int st = launch_raytrace<false>(b, ra, s);
    if (st) return st;
  }
  JSC_LAUNCH_CHECK();
  {
    const int st = launch_scan(b, ra.nlos, nr, (int64_t *)ra.los_off, s);
    if (st) return st;
  }
  // The LOS buffer is sized from the counting pass (one small copy).
  if (b->fixed) {
    // Fixed capacity (graph capture): no read-back, the buffers hold
    // max_seg points and the storing passes flag an overflow.
    *b->h_total = 0;
  } else {
    JSC_CUDA_TRY(cudaMemcpyAsync(b->h_total, ra.los_off + nr, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, s));
    JSC_CUDA_TRY(cudaStreamSynchronize(s));
  }
  if (b->fixed && (b->depth > 1 || (b->depth == 1 && b->fx_rounds < 1) ||
                   (refine && b->max_seg_b < b->max_seg))) {
    jsc_set_error(JSC_ERR_UNSUPPORTED,
                  "fixed-capacity runs cover clear air, aerosol extinction and single "
                  "scattering prepared by jsc_batch_set_fixed");
    return JSC_ERR_UNSUPPORTED;
  }
  if (refine) {
    if (*b->h_total > b->max_seg_b) {
      int st = batch_alloc_los_b(b, *b->h_total + *b->h_total / 4 + 1024);
      if (st) return st;
    }
    ra.geo = b->d_geo_b;
    ra.pts = b->d_pts_b;
    ra.max_seg = b->max_seg_b;
  } else {
    if (*b->h_total > b->max_seg) {
      int st = batch_alloc_los(b, *b->h_total + *b->h_total / 4 + 1024);
      if (st) return st;
    }
    b->n_points = b->fixed ? b->max_seg : *b->h_total;
    ra.geo = b->d_geo;
    ra.pts = b->d_pts;
    ra.max_seg = b->max_seg;
  }
  {
    const int st = launch_raytrace<true>(b, ra, s);
    if (st) return st;
  }
  JSC_LAUNCH_CHECK();
  if (refine) {
    if (b->fixed) {  // keep the refinement's reads inside the base buffer
      clamp_los_kernel<<<(nr + 127) / 128, 128, 0, s>>>(b->d_nlos_b, b->d_los_off_b, nr,
                                                         b->max_seg_b);
      JSC_LAUNCH_CHECK();
    }
    // Layer-edge points, chord steps and aerosol factors
    // (add_aerosol_layers, src/lineofsight.c:193-372).
    RefineArgs fa;
    memset(&fa, 0, sizeof(fa));
    fa.n_rays = nr;
    fa.ng = b->cfg.ng;
    fa.nw = b->cfg.nw;
    fa.W = b->W;
    fa.n_levels = b->n_levels;
    fa.ig_h2o = m->dv.ig_h2o;
    fa.ray_atm = b->d_ray_atm;
    fa.atm_off = b->d_atm_off;
    fa.z = b->d_z;
    fa.p = b->d_p;
    fa.t = b->d_t;
    fa.q = b->d_q;
    fa.k = b->d_k;
    fa.nlos_b = b->d_nlos_b;
    fa.off_b = b->d_los_off_b;
    fa.geo_b = b->d_geo_b;
    fa.pts_b = b->d_pts_b;
    fa.nlos = b->d_nlos;
    fa.off = b->d_los_off;
    fa.nl = b->aero_nl;
    fa.n_alti = b->n_alti;
    fa.altimax = b->altimax;
    fa.altimin = b->altimin;
    fa.transs = b->cfg.transs;
    fa.top = b->d_aero;
    fa.bottom = b->d_aero + NLMAX;
    fa.trans = b->d_aero + 2 * NLMAX;
    fa.alti = b->d_aero + 3 * NLMAX;
    fa.grid_np = ra.grid_np;
    fa.grid_p = ra.grid_p;
    fa.grid_t = ra.grid_t;
    fa.grid_nt = ra.grid_nt;
    fa.status = b->d_status;
    fa.geo = b->d_geo;
    fa.pts = b->d_pts;
    fa.max_seg = b->max_seg;
    refine_count_kernel<<<(nr + 127) / 128, 128, 0, s>>>(fa);
    JSC_LAUNCH_CHECK();
    {
      const int st = launch_scan(b, b->d_nlos, nr, b->d_los_off, s);
      if (st) return st;
    }
    if (b->fixed) {
      *b->h_total = 0;
    } else {
      JSC_CUDA_TRY(cudaMemcpyAsync(b->h_total, b->d_los_off + nr, sizeof(int64_t),
                                   cudaMemcpyDeviceToHost, s));
      JSC_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (*b->h_total > b->max_seg) {
      int st = batch_alloc_los(b, *b->h_total + *b->h_total / 4 + 1024);
      if (st) return st;
    }
    b->n_points = b->fixed ? b->max_seg : *b->h_total;
    fa.geo = b->d_geo;
    fa.pts = b->d_pts;
    fa.max_seg = b->max_seg;
    fa.ip = b->ip;
    fa.n_prof = b->n_atm;
    fa.psurf = b->d_psurf;
    fa.lat = b->d_lat;
    fa.cz = b->cz;
    fa.cx = b->cx;
    {
      const unsigned g = (unsigned)(((int64_t)nr * 32 + 127) / 128);
      if (b->ip == 2) refine_store_kernel<2><<<g, 128, 0, s>>>(fa);
      else if (b->ip == 3) refine_store_kernel<3><<<g, 128, 0, s>>>(fa);
      else refine_store_kernel<<<g, 128, 0, s>>>(fa);
    }
    JSC_LAUNCH_CHECK();
  }
  if (b->fixed) {
    clamp_los_kernel<<<(nr + 127) / 128, 128, 0, s>>>(b->d_nlos, b->d_los_off, nr, b->max_seg);
    JSC_LAUNCH_CHECK();
  }
  ev_record(b, JSC_T_RAYTRACE, 1, s);

  // Scattering source at every scattering point (srcfunc_sca), from the
  // child batches of secondary and solar pencils.
  const bool scattering = b->depth > 0;
  if (scattering) {
    ev_record(b, JSC_T_SCATTER, 0, s);
    int st = scatter_sources(b, s);
    if (st) return st;
    ev_record(b, JSC_T_SCATTER, 1, s);
  }

  EgaArgs ea;
  ea.m = m->dv;
  ea.cfg = b->cfg;
  ea.n_rays = nr;
  ea.W = b->W;
  ea.single_grid = m->n_grid == 1;
  int ndp = 1;
  if (m->nd <= 32) {
    while (ndp < m->nd) ndp <<= 1;
  } else {
    ndp = (m->nd + 31) / 32 * 32;
  }
  ea.ndp = ndp;
  ea.nlos = b->d_nlos;
  ea.los_off = b->d_los_off;
  ea.pts = b->d_pts;
  ea.tsurf = b->d_tsurf;
  ea.rad = b->d_rad;
  ea.tau = b->d_tau;
  ea.counters = b->d_counters;
  ea.digest = b->digest ? b->d_digest : nullptr;
  ea.beta = b->d_beta;
  ea.aero_nl = b->aero_nl;
  ea.src_sca = (scattering && (b->n_sp > 0 || b->fixed)) ? b->d_src : nullptr;
  ea.sp_off = (scattering && (b->n_sp > 0 || b->fixed)) ? b->d_sp_off : nullptr;
  ea.beta_ctm = b->d_ctm;
  ea.src_pl = b->d_srcp;
  ea.order = nullptr;
  const int variant = run_variant(b);
  if (kEgaVariants[variant].ray && ray_warps(m->ng)) {
    int e = jsc_ray_order(nr, b->d_ray_atm, b->d_nlos, b->d_tsurf, b->d_tp, b->d_rkeys,
                          b->d_rorder, b->d_rtmp, b->rtmp_bytes, s);
    if (e) {
      jsc_set_error(JSC_ERR_CUDA, "ray order: %s", cudaGetErrorString((cudaError_t)e));
      return JSC_ERR_CUDA;
    }
    ea.order = b->d_rorder;
  }
  if (lane_variant(variant)) {
    // continuum extinction and Planck source per (LOS point, channel)
    CtmArgs ca;
    ca.m = m->dv;
    ca.cfg = b->cfg;
    ca.n_points = b->n_points;
    ca.W = b->W;
    ca.pts = b->d_pts;
    ca.beta = b->d_ctm;
    ca.src = b->d_srcp;
    ca.n_live = b->fixed ? b->d_los_off + nr : nullptr;
    ev_record(b, JSC_T_CTM, 0, s);
    jsc_ctm_src_launch(ca, s);
    JSC_LAUNCH_CHECK();
    ev_record(b, JSC_T_CTM, 1, s);
  }
  b->last_ega = ea;
  ev_record(b, JSC_T_EGA, 0, s);
  int st = launch_ega(ea, nr, ndp, m->ng, variant, s);
  if (st) return st;
  JSC_LAUNCH_CHECK();
  ev_record(b, JSC_T_EGA, 1, s);
  // LOS point total for the work counters.
  JSC_CUDA_TRY(cudaMemcpyAsync(b->d_counters, b->d_los_off + nr, sizeof(int64_t),
                               cudaMemcpyDeviceToDevice, s));
  return JSC_OK;
}

static int map_status(unsigned st) {
  if (st & JSC_DEV_ERR_OBSERVER) {
    jsc_set_error(JSC_ERR_OBSERVER, "Observer below surface!");
    return JSC_ERR_OBSERVER;
  }
  if (st & JSC_DEV_ERR_NLOS) {
    jsc_set_error(JSC_ERR_NLOS, "Too many LOS points!");
    return JSC_ERR_NLOS;
  }
  if (st & JSC_DEV_ERR_QUEUE) {
    jsc_set_error(JSC_ERR_QUEUE, "Too many queue items!");
    return JSC_ERR_QUEUE;
  }
  if (st & JSC_DEV_ERR_WATCHDOG) {
    jsc_set_error(JSC_ERR_WATCHDOG, "device wait gave up");
    return JSC_ERR_WATCHDOG;
  }
  return JSC_OK;
}

#define DCPY(dst, src, n, s)                                                 \
  JSC_CUDA_TRY(cudaMemcpyAsync((dst), (src), (size_t)(n) * sizeof(*(src)),   \
                               cudaMemcpyDeviceToHost, (cudaStream_t)(s)))

extern "C" int jsc_batch_download(jsc_batch *b, const jsc_batch_output *out,
                                  void *stream) {
  if (!b || !out) return JSC_ERR_ARG;
  const int nr = b->n_rays, nd = b->cfg.nd;
  unsigned status = 0;
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  if (nr > 0) {
    if (out->rad) DCPY(out->rad, b->d_rad, (size_t)nr * nd, stream);
    if (out->tau) DCPY(out->tau, b->d_tau, (size_t)nr * nd, stream);
    if (out->tpz) DCPY(out->tpz, b->d_tp, nr, stream);
    if (out->tplon) DCPY(out->tplon, b->d_tp + nr, nr, stream);
    if (out->tplat) DCPY(out->tplat, b->d_tp + 2 * (size_t)nr, nr, stream);
    if (out->nlos) DCPY(out->nlos, b->d_nlos, nr, stream);
  }
  DCPY(&status, b->d_status, 1, stream);
  JSC_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  return map_status(status);
}

extern "C" int jsc_formod_batch(jsc_model *m, const ctl_t *ctl,
                                const jsc_batch_input *in,
                                const jsc_batch_output *out, void *stream) {
  jsc_batch *b = nullptr;
  int st = jsc_batch_create(m, ctl, in->n_atm, in->n_levels,
                            in->n_rays > 0 ? in->n_rays : 1, 0, &b);
  if (!st) st = jsc_batch_upload(b, in, stream);
  if (!st) st = jsc_batch_run(b, stream);
  if (!st) st = jsc_batch_download(b, out, stream);
  jsc_batch_destroy(b);
  return st;
}

extern "C" int jsc_batch_set_digest(jsc_batch *b, int on) {
  if (!b) return JSC_ERR_ARG;
  if (on && !b->d_digest) {
    int st = jsc_dmalloc(&b->d_digest, (size_t)b->max_rays * b->cfg.nd);
    if (st) return st;
  }
  b->digest = on;
  return JSC_OK;
}

extern "C" int jsc_batch_index_digest(jsc_batch *b, uint64_t *out) {
  if (!b || !out || !b->digest) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaMemcpy(out, b->d_digest,
                          (size_t)b->n_rays * b->cfg.nd * sizeof(uint64_t),
                          cudaMemcpyDeviceToHost));
  return JSC_OK;
}

extern "C" int jsc_batch_autotune(jsc_batch *b, void *stream) {
  if (!b || b->n_rays < 1) return JSC_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  b->ega_variant = kLaneBase;  // a lane variant also fills the continuum arrays
  int st = jsc_batch_run(b, stream);  // LOS records for the timing runs
  if (st) return st;
  EgaArgs ea = b->last_ega;
  ea.digest = nullptr;
  if (ray_warps(b->m->ng)) {
    int e = jsc_ray_order(b->n_rays, b->d_ray_atm, b->d_nlos, b->d_tsurf, b->d_tp, b->d_rkeys,
                          b->d_rorder, b->d_rtmp, b->rtmp_bytes, s);
    if (e) {
      jsc_set_error(JSC_ERR_CUDA, "ray order: %s", cudaGetErrorString((cudaError_t)e));
      return JSC_ERR_CUDA;
    }
    ea.order = b->d_rorder;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  JSC_CUDA_TRY(cudaEventCreate(&e0));
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    jsc_set_error(JSC_ERR_CUDA, "autotune: cudaEventCreate failed");
    return JSC_ERR_CUDA;
  }
  int best = kEgaDefault;
  float best_ms = 1e30f;
  for (int v = 0; v < kNumEgaVariants && !st; v++) {
    cudaError_t e = cudaEventRecord(e0, s);
    if (e == cudaSuccess) st = launch_ega(ea, b->n_rays, ea.ndp, b->m->ng, v, s);
    if (!st && e == cudaSuccess) e = cudaEventRecord(e1, s);
    if (!st && e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = -1;
    if (!st && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (!st && e != cudaSuccess) {
      jsc_set_error(JSC_ERR_CUDA, "autotune variant %d: %s", v, cudaGetErrorString(e));
      st = JSC_ERR_CUDA;
    }
    b->ega_variant_ms[v] = ms;
    if (!st && ms < best_ms) {
      best_ms = ms;
      best = v;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st) return st;
  b->ega_variant = best;
  return JSC_OK;
}

extern "C" int jsc_batch_set_variant(jsc_batch *b, int variant) {
  if (!b || variant < -1 || variant >= kNumEgaVariants) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_variant: variant %d outside -1..%d", variant,
                  kNumEgaVariants - 1);
    return JSC_ERR_ARG;
  }
  b->ega_variant = variant;
  return JSC_OK;
}

extern "C" double jsc_batch_variant_ms(const jsc_batch *b, int variant) {
  if (!b || variant < 0 || variant >= kNumEgaVariants) return -1;
  return b->ega_variant_ms[variant];
}

extern "C" int jsc_batch_variant(const jsc_batch *b, int *variant, int *blk, int *minb) {
  if (!b) return JSC_ERR_ARG;
  const int v = run_variant(b);
  if (variant) *variant = v;
  const int rw = kEgaVariants[v].ray ? ray_warps(b->m->ng) : 0;
  if (blk)
    *blk = kEgaVariants[v].ray
               ? (rw ? 32 * (rw + (kEgaVariants[v].ray == 1)) : kEgaVariants[kLaneBase + 4].blk)
               : kEgaVariants[v].blk;
  if (minb) *minb = kEgaVariants[v].ray && !rw ? kEgaVariants[kLaneBase + 4].minb
                                               : kEgaVariants[v].minb;
  return JSC_OK;
}

extern "C" void jsc_batch_set_timing(jsc_batch *b, int on) {
  if (b) b->timing = on;
}

extern "C" double jsc_batch_kernel_ms(const jsc_batch *b, const char *kernel) {
  if (!b || !b->timing || !kernel) return -1;
  int k = -1;
  if (!strcmp(kernel, "hydrostatic")) k = JSC_T_HYDRO;
  else if (!strcmp(kernel, "scatter")) k = JSC_T_SCATTER;
  else if (!strcmp(kernel, "continua")) k = JSC_T_CTM;
  else if (!strcmp(kernel, "surrogate")) k = JSC_T_SUR;
  else if (!strcmp(kernel, "raytrace")) k = JSC_T_RAYTRACE;
  else if (!strcmp(kernel, "ega_rt")) k = JSC_T_EGA;
  if (k < 0 || !b->ran[k]) return -1;
  float ms = -1;
  if (cudaEventSynchronize(b->ev[2 * k + 1]) != cudaSuccess) return -1;
  if (cudaEventElapsedTime(&ms, b->ev[2 * k], b->ev[2 * k + 1]) != cudaSuccess) return -1;
  return ms;
}

extern "C" int jsc_batch_counters(const jsc_batch *b, int64_t *n_points,
                                  int64_t *n_ega) {
  if (!b) return JSC_ERR_ARG;
  unsigned long long c[2] = {0, 0};
  JSC_CUDA_TRY(cudaMemcpy(c, b->d_counters, sizeof(c), cudaMemcpyDeviceToHost));
  if (n_points) *n_points = (int64_t)c[0];
  if (n_ega) *n_ega = (int64_t)c[1];
  return JSC_OK;
}

extern "C" int jsc_batch_set_surrogate(jsc_batch *b, jsc_surrogate *s, double tol_rel,
                                       int check_stride) {
  if (!b || (s && (jsc_sur_nout(s) != b->cfg.nd || tol_rel <= 0 || check_stride < 0))) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_surrogate: channel count, tolerance or stride");
    return JSC_ERR_ARG;
  }
  b->sur = s;
  b->sur_on = s != nullptr;
  b->sur_tol = (float)tol_rel;
  b->sur_stride = check_stride;
  return JSC_OK;
}

extern "C" int jsc_batch_set_surrogate_depth(jsc_batch *b, int depth, jsc_surrogate *s,
                                             double tol_rel, int check_stride) {
  if (!b || depth < 1 || depth > b->depth || depth > JSC_MAX_DEPTH) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_surrogate_depth: depth %d outside 1..%d", depth,
                  b ? b->depth : 0);
    return JSC_ERR_ARG;
  }
  if (depth == b->depth) return jsc_batch_set_surrogate(b, s, tol_rel, check_stride);
  if (s && (jsc_sur_nout(s) != b->cfg.nd || tol_rel <= 0 || check_stride < 0)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_set_surrogate_depth: channel count, tolerance or stride");
    return JSC_ERR_ARG;
  }
  b->sur_at[depth] = s;
  b->sur_tol_at[depth] = (float)tol_rel;
  b->sur_stride_at[depth] = check_stride;
  for (jsc_batch *c = b->child; c; c = c->child) {
    c->sur_at[depth] = s;
    c->sur_tol_at[depth] = (float)tol_rel;
    c->sur_stride_at[depth] = check_stride;
    if (c->depth == depth) {
      c->sur = s;
      c->sur_on = s != nullptr;
      c->sur_tol = (float)tol_rel;
      c->sur_stride = check_stride;
    }
  }
  return JSC_OK;
}

// The batch of the last run at scattering depth `depth` (b or a child).
static jsc_batch *batch_at_depth(jsc_batch *b, int depth) {
  for (jsc_batch *c = b; c; c = c->child)
    if (c->depth == depth) return c;
  return nullptr;
}

extern "C" int jsc_batch_scatter_samples_depth(jsc_batch *b, int depth, float *feat, double *src,
                                               int64_t max, int64_t *n) {
  jsc_batch *c = b ? batch_at_depth(b, depth) : nullptr;
  if (!c || !n) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_scatter_samples_depth: no batch of depth %d", depth);
    return JSC_ERR_ARG;
  }
  return jsc_batch_scatter_samples(c, feat, src, max, n);
}

extern "C" int jsc_batch_surrogate_stats_depth(const jsc_batch *b, int depth, int64_t *points,
                                               int64_t *fallback, int64_t *checked,
                                               double *max_rel_err, double *mean_rel_err,
                                               int *used) {
  jsc_batch *c = b ? batch_at_depth(const_cast<jsc_batch *>(b), depth) : nullptr;
  if (!c) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_surrogate_stats_depth: no batch of depth %d", depth);
    return JSC_ERR_ARG;
  }
  if (mean_rel_err) *mean_rel_err = c->sur_errn > 0 ? c->sur_errsum / (double)c->sur_errn : 0.0;
  return jsc_batch_surrogate_stats(c, points, fallback, checked, max_rel_err, used);
}

extern "C" int jsc_batch_surrogate_stats(const jsc_batch *b, int64_t *points, int64_t *fallback,
                                         int64_t *checked, double *max_rel_err, int *used) {
  if (!b) return JSC_ERR_ARG;
  if (points) *points = b->sur_points;
  if (fallback) *fallback = b->sur_fallback;
  if (checked) *checked = b->sur_checked;
  if (max_rel_err) *max_rel_err = b->sur_maxerr;
  // used: every chunk of the last run took its sources from the surrogate
  if (used) *used = b->sur_runs > 0 && b->sur_used_runs == b->sur_runs;
  return JSC_OK;
}

extern "C" int jsc_batch_scatter_samples(jsc_batch *b, float *feat, double *src, int64_t max,
                                         int64_t *n) {
  if (!b || !n) return JSC_ERR_ARG;
  *n = b->n_sp;
  if (!feat || !src || b->n_sp == 0) return JSC_OK;
  if (b->n_sp > max) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_scatter_samples: %lld points, room for %lld",
                  (long long)b->n_sp, (long long)max);
    return JSC_ERR_ARG;
  }
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  JSC_CUDA_TRY(cudaDeviceSynchronize());  // the last run may be on any stream
  float *d_f = nullptr;
  int st = jsc_dmalloc(&d_f, (size_t)b->n_sp * SUR_NF);
  if (st) return st;
  st = jsc_sur_features((int)b->n_sp, b->d_sp, d_f, 0);
  if (!st && cudaMemcpy(feat, d_f, (size_t)b->n_sp * SUR_NF * sizeof(float),
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    st = JSC_ERR_CUDA;
  if (!st && cudaMemcpy(src, b->d_src, (size_t)b->n_sp * b->cfg.nd * sizeof(double),
                        cudaMemcpyDeviceToHost) != cudaSuccess)
    st = JSC_ERR_CUDA;
  cudaFree(d_f);
  return st;
}

extern "C" int jsc_batch_set_fixed(jsc_batch *b, int on) {
  if (!b) return JSC_ERR_ARG;
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  if (on) {
    int st;
    if (b->depth > 0 && (st = prepare_fixed_scattering(b))) return st;
    if (b->cfg.sca_n > 0 && b->max_seg_b < b->max_seg &&
        (st = batch_alloc_los_b(b, b->max_seg)))
      return st;
    if (!b->h_status && cudaMallocHost((void **)&b->h_status, sizeof(unsigned)) != cudaSuccess) {
      jsc_set_error(JSC_ERR_NOMEM, "pinned host allocation");
      return JSC_ERR_NOMEM;
    }
    *b->h_status = 0;
  }
  b->fixed = on != 0;
  return JSC_OK;
}

extern "C" int jsc_batch_download_async(jsc_batch *b, const jsc_batch_output *out,
                                        void *stream) {
  if (!b || !out || !b->h_status) return JSC_ERR_ARG;
  const int nr = b->n_rays, nd = b->cfg.nd;
  if (nr > 0) {
    if (out->rad) DCPY(out->rad, b->d_rad, (size_t)nr * nd, stream);
    if (out->tau) DCPY(out->tau, b->d_tau, (size_t)nr * nd, stream);
    if (out->tpz) DCPY(out->tpz, b->d_tp, nr, stream);
    if (out->tplon) DCPY(out->tplon, b->d_tp + nr, nr, stream);
    if (out->tplat) DCPY(out->tplat, b->d_tp + 2 * (size_t)nr, nr, stream);
    if (out->nlos) DCPY(out->nlos, b->d_nlos, nr, stream);
  }
  DCPY(b->h_status, b->d_status, 1, stream);
  return JSC_OK;
}

extern "C" int jsc_batch_async_status(const jsc_batch *b) {
  if (!b || !b->h_status) return JSC_ERR_ARG;
  return map_status(*b->h_status);
}

// Host checks of the indices the kernels follow (as in jsc_batch_upload).
static int check_input(const jsc_batch *b, const jsc_batch_input *in) {
  if (in->n_atm < 1 || in->n_atm > b->max_atm || in->n_levels < 2 ||
      in->n_levels > b->max_levels || in->n_rays < 0 || in->n_rays > b->max_rays ||
      in->atm_off[0] != 0 || in->atm_off[in->n_atm] != in->n_levels) {
    jsc_set_error(JSC_ERR_ARG, "batch input exceeds the batch capacity or has bad offsets");
    return JSC_ERR_ARG;
  }
  for (int a = 0; a < in->n_atm; a++)
    if (in->atm_off[a + 1] - in->atm_off[a] < 2) {
      jsc_set_error(JSC_ERR_ARG, "profile %d has fewer than 2 levels", a);
      return JSC_ERR_ARG;
    }
  for (int r = 0; r < in->n_rays; r++)
    if (in->ray_atm[r] < 0 || in->ray_atm[r] >= in->n_atm) {
      jsc_set_error(JSC_ERR_ARG, "ray %d names profile %d of %d", r, in->ray_atm[r], in->n_atm);
      return JSC_ERR_ARG;
    }
  return JSC_OK;
}

extern "C" int jsc_batch_graph_capture(jsc_batch *b, const jsc_batch_input *in,
                                       const jsc_batch_output *out, void *stream) {
  if (!b || !in || !out || !stream || !b->fixed) {
    jsc_set_error(JSC_ERR_ARG, "jsc_batch_graph_capture: needs a fixed-capacity batch and a "
                               "non-default stream");
    return JSC_ERR_ARG;
  }
  int st = check_input(b, in);
  if (st) return st;
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  if (b->gexec) {
    cudaGraphExecDestroy(b->gexec);
    b->gexec = nullptr;
  }
  b->graph_ready = 0;
  cudaStream_t s = (cudaStream_t)stream;
  (void)cudaGetLastError();
  JSC_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  st = jsc_batch_upload(b, in, stream);
  if (!st) st = batch_run(b, s);
  if (!st) st = jsc_batch_download_async(b, out, stream);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (!st && e != cudaSuccess) {
    jsc_set_error(JSC_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    st = JSC_ERR_CUDA;
  }
  if (!st) {
    size_t nn = 0;
    b->graph_kernels = 0;
    if (cudaGraphGetNodes(g, nullptr, &nn) == cudaSuccess && nn > 0) {
      cudaGraphNode_t *nodes = (cudaGraphNode_t *)malloc(nn * sizeof(cudaGraphNode_t));
      if (nodes && cudaGraphGetNodes(g, nodes, &nn) == cudaSuccess)
        for (size_t i = 0; i < nn; i++) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel)
            b->graph_kernels++;
        }
      free(nodes);
    }
    e = cudaGraphInstantiate(&b->gexec, g, 0);
    if (e != cudaSuccess) {
      jsc_set_error(JSC_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
      st = JSC_ERR_CUDA;
      b->gexec = nullptr;
    }
  }
  if (g) cudaGraphDestroy(g);
  if (st) return st;
  b->gin = *in;
  b->graph_ready = 1;
  return JSC_OK;
}

extern "C" int jsc_batch_graph_launch(jsc_batch *b, void *stream) {
  if (!b || !b->graph_ready) return JSC_ERR_ARG;
  // the graph copies from the captured host arrays: check what they hold now
  int st = check_input(b, &b->gin);
  if (st) return st;
  JSC_CUDA_TRY(cudaSetDevice(b->m->device));
  JSC_CUDA_TRY(cudaGraphLaunch(b->gexec, (cudaStream_t)stream));
  for (int i = 0; i < b->graph_kernels; i++) jsc_count_launch();
  return JSC_OK;
}
