// Model upload: packs the host tables into the device layout.
//
// Device layout (all in HBM, read-only during a forward model):
//  * (p, T) grids, deduplicated across tables (most table sets share one);
//  * a row descriptor per (p level, T, emitter, channel) slot;
//  * one 8-byte node per table point (u, eps): a lookup reads the two
//    nodes of its interval and computes the slope with the same IEEE
//    single-precision operations the reference's LIN evaluates;
//  * Planck source tables with slopes, continuum coefficients per channel.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <vector>

#include "cuda_util.cuh"
#include "jsc_model.h"

static std::atomic<uint64_t> g_launches{0};
extern "C" void jsc_count_launch(void) { g_launches.fetch_add(1); }
extern "C" uint64_t jsc_launch_count(void) { return g_launches.load(); }

// One warp per row slot builds the row's nodes and sets the row's
// JSC_ROW_STRICT flag when u and eps both increase strictly along it.
__global__ void build_nodes_kernel(jsc_row *rows, const int64_t *row_pt,
                                   int nrows, const float *u, const float *e,
                                   jsc_node *nodes) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int r = warp; r < nrows; r += nwarps) {
    const int n = rows[r].nf & 0xffff;
    const int64_t pt = row_pt[r];
    const int off = rows[r].off;
    bool inc = true;
    for (int k = lane; k < n; k += 32) {
      jsc_node v;
      v.u = u[pt + k];
      v.e = e[pt + k];
      if (n >= 2) nodes[off + k] = v;
      if (k + 1 < n && (!(v.u < u[pt + k + 1]) || !(v.e < e[pt + k + 1]))) inc = false;
    }
    if (__all_sync(0xffffffffu, inc) && lane == 0) rows[r].nf |= JSC_ROW_STRICT << 16;
  }
}

static uint64_t fnv1a(const void *data, size_t n, uint64_t h) {
  const unsigned char *p = (const unsigned char *)data;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

static uint64_t grid_hash(const jsc_host_table *t) {
  uint64_t h = 1469598103934665603ull;
  h = fnv1a(&t->np, sizeof(int), h);
  h = fnv1a(t->p, sizeof(double) * (size_t)t->np, h);
  h = fnv1a(t->nt, sizeof(int) * (size_t)t->np, h);
  for (int ip = 0; ip < t->np; ip++)
    h = fnv1a(t->t[ip], sizeof(double) * (size_t)t->nt[ip], h);
  return h;
}

static bool grid_equal(const jsc_host_table *a, const jsc_host_table *b) {
  if (a->np != b->np) return false;
  if (memcmp(a->p, b->p, sizeof(double) * (size_t)a->np)) return false;
  if (memcmp(a->nt, b->nt, sizeof(int) * (size_t)a->np)) return false;
  for (int ip = 0; ip < a->np; ip++)
    if (memcmp(a->t[ip], b->t[ip], sizeof(double) * (size_t)a->nt[ip]))
      return false;
  return true;
}

template <typename T>
static int upload(T **dst, const T *src, size_t n) {
  int st = jsc_dmalloc(dst, n);
  if (st) return st;
  if (n) JSC_CUDA_TRY(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return JSC_OK;
}

static int model_upload(jsc_model *m, const jsc_host_model *hm) {
  const int ng = hm->ng, nd = hm->nd, ntab = ng * nd;
  const jsc_host_tables *ht = &hm->tables;
  const size_t slots_per_tab = (size_t)TBLNPMAX * TBLNTMAX;
  const size_t nslots = (size_t)ntab * slots_per_tab;

  // Deduplicate (p, T) grids.
  std::vector<int> tab_grid(ntab > 0 ? ntab : 1, -1);
  std::vector<int> grid_rep;             // representative table per grid
  std::vector<uint64_t> grid_h;
  for (int ti = 0; ti < ntab; ti++) {
    const jsc_host_table *t = &ht->tab[ti];
    if (t->np < 2) continue;
    uint64_t h = grid_hash(t);
    int found = -1;
    for (size_t g = 0; g < grid_rep.size(); g++)
      if (grid_h[g] == h && grid_equal(&ht->tab[grid_rep[g]], t)) {
        found = (int)g;
        break;
      }
    if (found < 0) {
      found = (int)grid_rep.size();
      grid_rep.push_back(ti);
      grid_h.push_back(h);
    }
    tab_grid[ti] = found;
  }
  const int ngrid = (int)grid_rep.size();
  std::vector<int> g_np(ngrid > 0 ? ngrid : 1, 0);
  std::vector<double> g_p((size_t)(ngrid > 0 ? ngrid : 1) * TBLNPMAX, 0.0);
  std::vector<int> g_nt((size_t)(ngrid > 0 ? ngrid : 1) * TBLNPMAX, 0);
  std::vector<double> g_t((size_t)(ngrid > 0 ? ngrid : 1) * TBLNPMAX * TBLNTMAX, 0.0);
  for (int g = 0; g < ngrid; g++) {
    const jsc_host_table *t = &ht->tab[grid_rep[g]];
    g_np[g] = t->np;
    for (int ip = 0; ip < t->np; ip++) {
      g_p[(size_t)g * TBLNPMAX + ip] = t->p[ip];
      g_nt[(size_t)g * TBLNPMAX + ip] = t->nt[ip];
      for (int it = 0; it < t->nt[ip]; it++)
        g_t[((size_t)g * TBLNPMAX + ip) * TBLNTMAX + it] = t->t[ip][it];
    }
  }

  // Row descriptors and node offsets, ordered (p level, temperature,
  // emitter, channel): the threads of a warp (neighbouring channels) look
  // up the same (p, T) node of the same emitter at the same time, so their
  // descriptors are contiguous and their nodes lie within a few hundred KB.
  std::vector<jsc_row> rows(nslots > 0 ? nslots : 1);
  std::vector<int64_t> row_pt(nslots > 0 ? nslots : 1, 0);
  int64_t niv = 0;
  for (int ip = 0; ip < TBLNPMAX; ip++)
    for (int it = 0; it < TBLNTMAX; it++)
      for (int ig = 0; ig < ng; ig++)
        for (int id = 0; id < nd; id++) {
          const int ti = id * ng + ig;
          const jsc_host_table *t = &ht->tab[ti];
          size_t s = (((size_t)ip * TBLNTMAX + it) * ng + ig) * nd + id;
          rows[s].off = 0;
          rows[s].nf = 0;
          if (t->np < 2 || ip >= t->np || it >= t->nt[ip]) continue;
          int n = t->nu[ip][it];
          if (n < 0) n = 0;
          int64_t pt = t->off[ip][it];
          rows[s].off = (int)niv;
          rows[s].nf = n;  /* build_nodes_kernel adds the strictness flag */
          row_pt[s] = pt;
          if (n >= 2) niv += n;
          if (niv > 0x7fffffff) {
            jsc_set_error(JSC_ERR_TABLE, "emissivity tables exceed 2^31 points");
            return JSC_ERR_TABLE;
          }
        }

  int st;
  if ((st = upload(&m->d_grid_np, g_np.data(), g_np.size()))) return st;
  if ((st = upload(&m->d_grid_p, g_p.data(), g_p.size()))) return st;
  if ((st = upload(&m->d_grid_nt, g_nt.data(), g_nt.size()))) return st;
  if ((st = upload(&m->d_grid_t, g_t.data(), g_t.size()))) return st;
  if ((st = upload(&m->d_tab_grid, tab_grid.data(), tab_grid.size()))) return st;
  if ((st = upload(&m->d_rows, rows.data(), rows.size()))) return st;
  if ((st = jsc_dmalloc(&m->d_nodes, (size_t)niv))) return st;
  m->n_nodes = niv;
  m->n_grid = ngrid;
  m->grid_np0 = g_np.empty() ? 0 : g_np[0];

  if (niv > 0) {
    float *du = nullptr, *de = nullptr;
    int64_t *drp = nullptr;
    if ((st = upload(&du, ht->u, (size_t)ht->n_points))) return st;
    if ((st = upload(&de, ht->eps, (size_t)ht->n_points))) return st;
    if ((st = upload(&drp, row_pt.data(), row_pt.size()))) return st;
    build_nodes_kernel<<<148 * 8, 256>>>(m->d_rows, drp, (int)nslots, du, de,
                                          m->d_nodes);
    jsc_count_launch();
    cudaError_t e = cudaDeviceSynchronize();
    cudaFree(du);
    cudaFree(de);
    cudaFree(drp);
    if (e != cudaSuccess) {
      jsc_set_error(JSC_ERR_CUDA, "build_nodes: %s", cudaGetErrorString(e));
      return JSC_ERR_CUDA;
    }
  }

  const size_t npl = (size_t)nd * JSC_NPLANCK;
  if ((st = upload(&m->d_planck_b, hm->planck_b, npl))) return st;
  if ((st = upload(&m->d_planck_s, hm->planck_s, npl))) return st;
  if ((st = upload(&m->d_ctm, hm->ctm, (size_t)nd))) return st;
  if ((st = upload(&m->d_nu, hm->nu, (size_t)nd))) return st;
  if ((st = upload(&m->d_window, hm->window, (size_t)nd))) return st;

  m->table_bytes = (size_t)niv * sizeof(jsc_node) + rows.size() * sizeof(jsc_row);

  jsc_dev_model &d = m->dv;
  d.ng = ng;
  d.nd = nd;
  d.nw = hm->nw;
  d.ig_co2 = hm->ig_co2;
  d.ig_h2o = hm->ig_h2o;
  d.n_grid = ngrid;
  d.grid_np = m->d_grid_np;
  d.grid_p = m->d_grid_p;
  d.grid_nt = m->d_grid_nt;
  d.grid_t = m->d_grid_t;
  d.tab_grid = m->d_tab_grid;
  d.rows = m->d_rows;
  d.nodes = m->d_nodes;
  d.planck_b = m->d_planck_b;
  d.planck_s = m->d_planck_s;
  d.ctm = m->d_ctm;
  d.nu = m->d_nu;
  d.window = m->d_window;
  return JSC_OK;
}

extern "C" int jsc_model_create(const ctl_t *ctl, int device, jsc_model **out) {
  if (!ctl || !out) {
    jsc_set_error(JSC_ERR_ARG, "jsc_model_create: NULL argument");
    return JSC_ERR_ARG;
  }
  *out = nullptr;
  JSC_CUDA_TRY(cudaSetDevice(device));
  jsc_host_model *hm = (jsc_host_model *)calloc(1, sizeof(jsc_host_model));
  jsc_model *m = (jsc_model *)calloc(1, sizeof(jsc_model));
  if (!hm || !m) {
    free(hm);
    free(m);
    jsc_set_error(JSC_ERR_NOMEM, "jsc_model_create: host allocation");
    return JSC_ERR_NOMEM;
  }
  int st = jsc_host_model_load(ctl, hm);
  if (!st) {
    m->device = device;
    m->ng = hm->ng;
    m->nd = hm->nd;
    m->nw = hm->nw;
    for (int id = 0; id < hm->nd; id++) m->nu[id] = hm->nu[id];
    st = model_upload(m, hm);
  }
  jsc_host_model_free(hm);
  free(hm);
  if (st) {
    jsc_model_destroy(m);
    return st;
  }
  *out = m;
  return JSC_OK;
}

extern "C" void jsc_model_destroy(jsc_model *m) {
  if (!m) return;
  cudaFree(m->d_grid_np);
  cudaFree(m->d_grid_p);
  cudaFree(m->d_grid_nt);
  cudaFree(m->d_grid_t);
  cudaFree(m->d_tab_grid);
  cudaFree(m->d_rows);
  cudaFree(m->d_nodes);
  cudaFree(m->d_planck_b);
  cudaFree(m->d_planck_s);
  cudaFree(m->d_ctm);
  cudaFree(m->d_nu);
  cudaFree(m->d_window);
  free(m);
}

extern "C" size_t jsc_model_table_bytes(const jsc_model *m) {
  return m ? m->table_bytes : 0;
}
