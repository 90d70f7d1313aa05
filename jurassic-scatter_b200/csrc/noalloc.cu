// jsc_formod_batch_noalloc: the clear-air batch forward model of
// jsc_formod_batch (same kernels, same launch order, same results) with every
// per-call device buffer carved from one static device array instead of
// cudaMalloc'd batch buffers.  The call allocates no device or host memory.
//
// Scratch: JSC_NOALLOC_SCRATCH_BYTES (64 MiB) per device, a file-scope
// __device__ array.  Its device address is looked up once per device with
// cudaGetSymbolAddress (the first call on a device does this, with that
// device current) and cached.  Each call lays out, 256-byte aligned:
//   inputs     atm_off, z, lon, lat, p (as given), t, q[ng], k[nw],
//              ray_atm, time/obsz/obslon/obslat/vpz/vplon/vplat
//   work       p after hydrostatic balance, zmin/zmax per profile,
//              nlos, los_off, tsurf, tangent points, status word, counters
//   outputs    rad, tau [n_rays][nd]
//   LOS        the rest: geo [4] + records [W] doubles per LOS point
// Only the status word and the two work counters must start at zero; they
// are cleared on the stream at the start of every call.  Everything else is
// written by a kernel or a copy before anything reads it.
#include <pthread.h>
#include <stdio.h>
#include <string.h>

#include "kernels.cuh"
#include "ega_kernel.cuh"

#define JSC_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char jsc_noalloc_scratch[JSC_NOALLOC_SCRATCH_BYTES];

static unsigned char *g_scratch[JSC_NOALLOC_MAX_DEVICES];
static pthread_mutex_t g_lock[JSC_NOALLOC_MAX_DEVICES];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

static void init_locks(void) {
  for (int i = 0; i < JSC_NOALLOC_MAX_DEVICES; i++) pthread_mutex_init(&g_lock[i], nullptr);
}

// Bump layout over the scratch; every region starts on a 256-byte boundary.
struct Carve {
  size_t off;
  template <typename T>
  T *take(unsigned char *base, size_t n) {
    T *p = (T *)(base + off);
    off += ((n > 0 ? n : 1) * sizeof(T) + 255) & ~(size_t)255;
    return p;
  }
};

#define NCPY(dst, src, n, s)                                                 \
  JSC_CUDA_TRY(cudaMemcpyAsync((dst), (src), (size_t)(n) * sizeof(*(src)),   \
                               cudaMemcpyHostToDevice, (s)))
#define NDCPY(dst, src, n, s)                                                \
  JSC_CUDA_TRY(cudaMemcpyAsync((dst), (src), (size_t)(n) * sizeof(*(src)),   \
                               cudaMemcpyDeviceToHost, (s)))

static int noalloc_run(jsc_model *m, const ctl_t *ctl, const jsc_batch_input *in,
                       const jsc_batch_output *out, cudaStream_t s,
                       unsigned char *base) {
  const int ng = ctl->ng, nw = ctl->nw, nd = ctl->nd;
  const int na = in->n_atm, nl = in->n_levels, nr = in->n_rays;
  const int W = JSC_REC_W(nw, ng);
  Carve c{0};
  int *d_atm_off = c.take<int>(base, (size_t)na + 1);
  double *d_z = c.take<double>(base, nl);
  double *d_lon = c.take<double>(base, nl);
  double *d_lat = c.take<double>(base, nl);
  double *d_p_in = c.take<double>(base, nl);
  double *d_t = c.take<double>(base, nl);
  double *d_q = c.take<double>(base, (size_t)nl * (ng > 0 ? ng : 1));
  double *d_k = c.take<double>(base, (size_t)nl * (nw > 0 ? nw : 1));
  double *d_p = c.take<double>(base, nl);
  double *d_zmin = c.take<double>(base, na);
  double *d_zmax = c.take<double>(base, na);
  int *d_ray_atm = c.take<int>(base, nr);
  double *d_ray = c.take<double>(base, (size_t)nr * 7);
  int *d_nlos = c.take<int>(base, nr);
  int64_t *d_los_off = c.take<int64_t>(base, (size_t)nr + 1);
  double *d_tsurf = c.take<double>(base, nr);
  double *d_tp = c.take<double>(base, (size_t)nr * 3);
  double *d_rad = c.take<double>(base, (size_t)nr * nd);
  double *d_tau = c.take<double>(base, (size_t)nr * nd);
  unsigned *d_status = c.take<unsigned>(base, 1);
  unsigned long long *d_counters = c.take<unsigned long long>(base, 2);
  const size_t fixed = c.off;
  const size_t per_point = (size_t)(4 + W) * sizeof(double);
  if (fixed + per_point > (size_t)JSC_NOALLOC_SCRATCH_BYTES) {
    jsc_set_error(JSC_ERR_ARG,
                  "jsc_formod_batch_noalloc: %d profiles, %d levels and %d rays need "
                  "%zu bytes of scratch before any LOS point; the static scratch holds %zu",
                  na, nl, nr, fixed + per_point, (size_t)JSC_NOALLOC_SCRATCH_BYTES);
    return JSC_ERR_ARG;
  }
  const int64_t max_seg = (int64_t)(((size_t)JSC_NOALLOC_SCRATCH_BYTES - fixed) / per_point);
  double *d_geo = c.take<double>(base, (size_t)max_seg * 4);
  double *d_pts = (double *)(base + c.off);  // the rest, max_seg * W doubles

  (void)cudaGetLastError();  // launch checks below report this call's errors only
  // Zero-start state: the status word (kernels OR error bits into it) and
  // the work counters (the EGA kernel adds to them).
  JSC_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(unsigned), s));
  JSC_CUDA_TRY(cudaMemsetAsync(d_counters, 0, 2 * sizeof(unsigned long long), s));

  NCPY(d_atm_off, in->atm_off, na + 1, s);
  NCPY(d_z, in->z, nl, s);
  NCPY(d_lon, in->lon, nl, s);
  NCPY(d_lat, in->lat, nl, s);
  NCPY(d_p_in, in->p, nl, s);
  NCPY(d_t, in->t, nl, s);
  if (ng > 0) NCPY(d_q, in->q, (size_t)ng * nl, s);
  if (nw > 0) NCPY(d_k, in->k, (size_t)nw * nl, s);
  if (nr > 0) {
    NCPY(d_ray_atm, in->ray_atm, nr, s);
    const double *cols[7] = {in->time, in->obsz, in->obslon, in->obslat,
                             in->vpz, in->vplon, in->vplat};
    for (int i = 0; i < 7; i++) {
      if (cols[i]) NCPY(d_ray + (size_t)i * nr, cols[i], nr, s);
      else JSC_CUDA_TRY(cudaMemsetAsync(d_ray + (size_t)i * nr, 0, (size_t)nr * sizeof(double), s));
    }
  }

  AtmArgs aa;
  aa.n_atm = na;
  aa.n_levels = nl;
  aa.ng = ng;
  aa.nw = nw;
  aa.ig_h2o = m->dv.ig_h2o;
  aa.off = d_atm_off;
  aa.z = d_z;
  aa.lon = d_lon;
  aa.lat = d_lat;
  aa.p_in = d_p_in;
  aa.t = d_t;
  aa.q = d_q;
  aa.k = d_k;
  aa.p = d_p;
  aa.zmin = d_zmin;
  aa.zmax = d_zmax;
  aa.hydz = ctl->hydz;
  hydro_kernel<<<(na + 127) / 128, 128, 0, s>>>(aa);
  JSC_LAUNCH_CHECK();

  unsigned status = 0;
  if (nr > 0) {
    RayArgs ra;
    ra.n_rays = nr;
    ra.ng = ng;
    ra.nw = nw;
    ra.ig_h2o = m->dv.ig_h2o;
    ra.n_levels = nl;
    ra.refrac = ctl->refrac;
    ra.rayds = ctl->rayds;
    ra.raydz = ctl->raydz;
    ra.ray_atm = d_ray_atm;
    ra.atm_off = d_atm_off;
    ra.time = d_ray;
    ra.obsz = d_ray + (size_t)nr;
    ra.obslon = d_ray + 2 * (size_t)nr;
    ra.obslat = d_ray + 3 * (size_t)nr;
    ra.vpz = d_ray + 4 * (size_t)nr;
    ra.vplon = d_ray + 5 * (size_t)nr;
    ra.vplat = d_ray + 6 * (size_t)nr;
    ra.z = d_z;
    ra.p = d_p;
    ra.t = d_t;
    ra.q = d_q;
    ra.k = d_k;
    ra.zmin = d_zmin;
    ra.zmax = d_zmax;
    ra.nlos = d_nlos;
    ra.los_off = d_los_off;
    ra.W = W;
    ra.tsurf = d_tsurf;
    ra.tp = d_tp;
    ra.status = d_status;
    ra.raw_q = 0;
    ra.geo = d_geo;
    ra.pts = d_pts;
    ra.max_seg = max_seg;
    ra.grid_np = 0;
    ra.grid_p = ra.grid_t = nullptr;
    ra.grid_nt = nullptr;
    raytrace_kernel<false><<<(nr + 127) / 128, 128, 0, s>>>(ra);
    JSC_LAUNCH_CHECK();
    scan_kernel<<<1, 1024, 0, s>>>(d_nlos, nr, d_los_off);
    JSC_LAUNCH_CHECK();
    // LOS point total of the counting pass, and the point count of the
    // shared (p, T) grid, read back in one wait on the stream.
    int64_t total = 0;
    int gnp = 0;
    NDCPY(&total, d_los_off + nr, 1, s);
    if (m->n_grid == 1) NDCPY(&gnp, m->d_grid_np, 1, s);
    JSC_CUDA_TRY(cudaStreamSynchronize(s));
    if (total > max_seg) {
      jsc_set_error(JSC_ERR_ARG,
                    "jsc_formod_batch_noalloc: the rays need %lld LOS points; the static "
                    "scratch holds %lld for this input (%zu bytes per point)",
                    (long long)total, (long long)max_seg, per_point);
      return JSC_ERR_ARG;
    }
    if (m->n_grid == 1) {
      ra.grid_np = gnp;
      ra.grid_p = m->d_grid_p;
      ra.grid_nt = m->d_grid_nt;
      ra.grid_t = m->d_grid_t;
    }
    raytrace_kernel<true><<<(nr + 127) / 128, 128, 0, s>>>(ra);
    JSC_LAUNCH_CHECK();

    EgaArgs ea;
    memset(&ea, 0, sizeof(ea));  // no scattering source, no digests
    ea.m = m->dv;
    jsc_run_cfg &cf = ea.cfg;
    memset(&cf, 0, sizeof(cf));
    cf.ng = ng;
    cf.nd = nd;
    cf.nw = nw;
    cf.ctm_co2 = ctl->ctm_co2;
    cf.ctm_h2o = ctl->ctm_h2o;
    cf.ctm_n2 = ctl->ctm_n2;
    cf.ctm_o2 = ctl->ctm_o2;
    cf.refrac = ctl->refrac;
    cf.rayds = ctl->rayds;
    cf.raydz = ctl->raydz;
    cf.hydz = ctl->hydz;
    cf.transs = ctl->transs;
    ea.n_rays = nr;
    ea.W = W;
    ea.single_grid = m->n_grid == 1;
    int ndp = 1;
    if (nd <= 32) {
      while (ndp < nd) ndp <<= 1;
    } else {
      ndp = (nd + 31) / 32 * 32;
    }
    ea.ndp = ndp;
    ea.nlos = d_nlos;
    ea.los_off = d_los_off;
    ea.pts = d_pts;
    ea.tsurf = d_tsurf;
    ea.rad = d_rad;
    ea.tau = d_tau;
    ea.counters = d_counters;
    ea.digest = nullptr;
    ea.beta = nullptr;
    ea.aero_nl = 0;
    const int64_t threads = (int64_t)nr * ndp;
    const unsigned g128 = (unsigned)((threads + 127) / 128);
    const unsigned g256 = (unsigned)((threads + 255) / 256);
    // The default launch variant of jsc_batch_run (every variant computes
    // the same operations in the same order; they differ in registers and
    // unrolling only).
    const int v = JSC_EGA_DEFAULT_VARIANT;
    if (ng <= 2) jsc_ega_launch_g2(ea, g128, g256, v, false, s);
    else if (ng <= 4) jsc_ega_launch_g4(ea, g128, g256, v, false, s);
    else if (ng <= 8) jsc_ega_launch_g8(ea, g128, g256, v, false, s);
    else jsc_ega_launch_gmax(ea, g128, g256, v, false, s);
    JSC_LAUNCH_CHECK();

    if (out->rad) NDCPY(out->rad, d_rad, (size_t)nr * nd, s);
    if (out->tau) NDCPY(out->tau, d_tau, (size_t)nr * nd, s);
    if (out->tpz) NDCPY(out->tpz, d_tp, nr, s);
    if (out->tplon) NDCPY(out->tplon, d_tp + nr, nr, s);
    if (out->tplat) NDCPY(out->tplat, d_tp + 2 * (size_t)nr, nr, s);
    if (out->nlos) NDCPY(out->nlos, d_nlos, nr, s);
  }
  NDCPY(&status, d_status, 1, s);
  JSC_CUDA_TRY(cudaStreamSynchronize(s));
  if (status & JSC_DEV_ERR_OBSERVER) {
    jsc_set_error(JSC_ERR_OBSERVER, "Observer below surface!");
    return JSC_ERR_OBSERVER;
  }
  if (status & JSC_DEV_ERR_NLOS) {
    jsc_set_error(JSC_ERR_NLOS, "Too many LOS points!");
    return JSC_ERR_NLOS;
  }
  return JSC_OK;
}

extern "C" int jsc_formod_batch_noalloc(jsc_model *m, const ctl_t *ctl,
                                        const jsc_batch_input *in,
                                        const jsc_batch_output *out, void *stream) {
  if (!m || !ctl || !in || !out) {
    jsc_set_error(JSC_ERR_ARG, "jsc_formod_batch_noalloc: null argument");
    return JSC_ERR_ARG;
  }
  if (ctl->ng != m->ng || ctl->nd != m->nd || ctl->nw != m->nw) {
    jsc_set_error(JSC_ERR_ARG, "jsc_formod_batch_noalloc: ctl does not match the model");
    return JSC_ERR_ARG;
  }
  if (ctl->ip != 1) {
    jsc_set_error(JSC_ERR_UNSUPPORTED, "only IP=1 (profile interpolation) runs on the GPU");
    return JSC_ERR_UNSUPPORTED;
  }
  if (ctl->sca_n > 0) {
    jsc_set_error(JSC_ERR_UNSUPPORTED,
                  "jsc_formod_batch_noalloc runs the clear-air path only (SCA_N = 0)");
    return JSC_ERR_UNSUPPORTED;
  }
  if (m->device < 0 || m->device >= JSC_NOALLOC_MAX_DEVICES) {
    jsc_set_error(JSC_ERR_ARG, "jsc_formod_batch_noalloc: device %d out of range", m->device);
    return JSC_ERR_ARG;
  }
  // The same input checks as jsc_batch_upload: every index a kernel follows
  // stays inside its buffer.
  if (in->n_atm < 1 || in->n_levels < 2 || in->n_rays < 0 || !in->atm_off ||
      !in->z || !in->lon || !in->lat || !in->p || !in->t ||
      (ctl->ng > 0 && !in->q) || (ctl->nw > 0 && !in->k) ||
      (in->n_rays > 0 && !in->ray_atm)) {
    jsc_set_error(JSC_ERR_ARG, "jsc_formod_batch_noalloc: invalid batch input");
    return JSC_ERR_ARG;
  }
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
      jsc_set_error(JSC_ERR_ARG, "ray %d names profile %d of %d", r, in->ray_atm[r], in->n_atm);
      return JSC_ERR_ARG;
    }
  pthread_once(&g_once, init_locks);
  const int dev = m->device;
  // One caller at a time per device: the scratch is shared by every call.
  pthread_mutex_lock(&g_lock[dev]);
  int st = JSC_OK;
  cudaError_t e = cudaSetDevice(dev);
  if (e == cudaSuccess && !g_scratch[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, jsc_noalloc_scratch);
    if (e == cudaSuccess) g_scratch[dev] = (unsigned char *)p;
  }
  if (e != cudaSuccess) {
    jsc_set_error(JSC_ERR_CUDA, "jsc_formod_batch_noalloc: scratch set-up on device %d: %s",
                  dev, cudaGetErrorString(e));
    st = JSC_ERR_CUDA;
  } else {
    st = noalloc_run(m, ctl, in, out, (cudaStream_t)stream, g_scratch[dev]);
    // A failed call may leave copies or kernels queued on its stream that
    // still write the scratch; wait for them before the next caller (on any
    // stream) gets the lock.  The wait's own error is not this call's.
    if (st != JSC_OK) (void)cudaStreamSynchronize((cudaStream_t)stream);
  }
  pthread_mutex_unlock(&g_lock[dev]);
  return st;
}
