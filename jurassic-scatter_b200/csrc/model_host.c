/*
 * Host-side model inputs: emissivity tables, filter functions, the Planck
 * source table and per-channel continuum coefficients.  Everything here runs
 * once per model (table set), before anything is uploaded to the GPU.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "jsc_internal.h"
#include "ckd_tables.h"

/* ------------------------------------------------------------------ errors */

static __thread int jsc_err_status = JSC_OK;
static __thread char jsc_err_msg[1024];

void jsc_set_error(int status, const char *fmt, ...) {
  va_list ap;
  jsc_err_status = status;
  va_start(ap, fmt);
  vsnprintf(jsc_err_msg, sizeof(jsc_err_msg), fmt, ap);
  va_end(ap);
}

const char *jsc_last_error_message(void) { return jsc_err_msg; }

const char *jsc_status_string(int status) {
  switch (status) {
    case JSC_OK: return "ok";
    case JSC_ERR_ARG: return "invalid argument";
    case JSC_ERR_CUDA: return "CUDA error";
    case JSC_ERR_FILE: return "cannot read input file";
    case JSC_ERR_TABLE: return "emissivity table exceeds a dimension";
    case JSC_ERR_NLOS: return "too many LOS points";
    case JSC_ERR_OBSERVER: return "observer below surface";
    case JSC_ERR_QUEUE: return "too many queue items";
    case JSC_ERR_WATCHDOG: return "device wait gave up";
    case JSC_ERR_UNSUPPORTED: return "feature not supported by the GPU path";
    case JSC_ERR_NOMEM: return "out of memory";
  }
  return "unknown status";
}

/* --------------------------------------------------- GSL 1.15 restatements */

/* gsl_expm1 (GSL 1.15 sys/expm1.c): Taylor series below ln 2, else
 * exp(x)-1.  Used by planck() so the source tables match the reference. */
double jsc_gsl_expm1(double x) {
  if (fabs(x) < M_LN2) {
    double i = 1.0, sum = x, term = x / 1.0;
    do {
      i++;
      term *= x / i;
      sum += term;
    } while (fabs(term) > fabs(sum) * 2.2204460492503131e-16);
    return sum;
  }
  return exp(x) - 1;
}

/* gsl_log1p (GSL 1.15 sys/log1p.c): log(1+x) with the rounding error of
 * 1+x compensated. */
double jsc_gsl_log1p(double x) {
  volatile double y, z;
  y = 1 + x;
  z = y - 1;
  return log(y) - (z - x) / y;
}

int jsc_find_emitter(const ctl_t *ctl, const char *name) {
  for (int ig = 0; ig < ctl->ng; ig++)
    if (strcasecmp(ctl->emitter[ig], name) == 0) return ig;
  return -1;
}

/* ------------------------------------------------------------ table files */

static int tables_reserve(jsc_host_tables *ht, int64_t extra) {
  if (ht->n_points + extra <= ht->cap_points) return JSC_OK;
  int64_t cap = ht->cap_points ? ht->cap_points : (1 << 20);
  while (cap < ht->n_points + extra) cap *= 2;
  float *u = (float *)realloc(ht->u, (size_t)cap * sizeof(float));
  if (!u) return JSC_ERR_NOMEM;
  ht->u = u;
  float *e = (float *)realloc(ht->eps, (size_t)cap * sizeof(float));
  if (!e) return JSC_ERR_NOMEM;
  ht->eps = e;
  ht->cap_points = cap;
  return JSC_OK;
}

#define RD(ptr, size, n, f) (fread((ptr), (size), (size_t)(n), (f)) == (size_t)(n))

/* Binary table, the layout written by the reference's tab2bin
 * (src/tab2bin.c:49-63) and read by read_tbl (src/forwardmodel.c:630-656). */
static int read_table_bin(FILE *in, const char *fn, jsc_host_tables *ht,
                          jsc_host_table *tb) {
  if (!RD(&tb->np, sizeof(int), 1, in)) goto bad;
  if (tb->np > TBLNPMAX) {
    jsc_set_error(JSC_ERR_TABLE, "Too many pressure levels in %s", fn);
    return JSC_ERR_TABLE;
  }
  if (tb->np < 0) tb->np = 0;
  if (!RD(tb->p, sizeof(double), tb->np, in)) goto bad;
  if (!RD(tb->nt, sizeof(int), tb->np, in)) goto bad;
  for (int ip = 0; ip < tb->np; ip++) {
    if (tb->nt[ip] > TBLNTMAX) {
      jsc_set_error(JSC_ERR_TABLE, "Too many temperatures in %s", fn);
      return JSC_ERR_TABLE;
    }
    if (tb->nt[ip] < 0) tb->nt[ip] = 0;
    if (!RD(tb->t[ip], sizeof(double), tb->nt[ip], in)) goto bad;
    if (!RD(tb->nu[ip], sizeof(int), tb->nt[ip], in)) goto bad;
    for (int it = 0; it < tb->nt[ip]; it++) {
      int n = tb->nu[ip][it];
      /* The reference reads min(n, TBLNUMAX) values but keeps n, which
       * misaligns the rest of the file; refuse such tables instead. */
      if (n > TBLNUMAX) {
        jsc_set_error(JSC_ERR_TABLE, "Too many column densities in %s", fn);
        return JSC_ERR_TABLE;
      }
      if (n < 0) n = tb->nu[ip][it] = 0;
      int st = tables_reserve(ht, n);
      if (st) return st;
      tb->off[ip][it] = ht->n_points;
      if (!RD(ht->u + ht->n_points, sizeof(float), n, in)) goto bad;
      if (!RD(ht->eps + ht->n_points, sizeof(float), n, in)) goto bad;
      ht->n_points += n;
    }
  }
  return JSC_OK;
bad:
  jsc_set_error(JSC_ERR_FILE, "Error while reading %s", fn);
  return JSC_ERR_FILE;
}

/* ASCII table "p T u eps" per line, read with the reference's rules
 * (src/forwardmodel.c:661-733): a new row starts when p or T changes; a
 * point is appended only if u and eps both increase, otherwise it replaces
 * the last point of the row; rows are capped at TBLNUMAX-1 accepted points. */
static int read_table_tab(FILE *in, const char *fn, jsc_host_tables *ht,
                          jsc_host_table *tb, float *ubuf, float *ebuf) {
  char line[LEN];
  double press, temp, u, eps;
  double eps_old = -999, press_old = -999, temp_old = -999, u_old = -999;
  int np = -1;
  static const size_t RS = TBLNUMAX;
  (void)fn;
  while (fgets(line, LEN, in)) {
    if (sscanf(line, "%lg %lg %lg %lg", &press, &temp, &u, &eps) != 4) continue;
    if (press != press_old) {
      press_old = press;
      if (++np >= TBLNPMAX) {
        jsc_set_error(JSC_ERR_TABLE, "Too many pressure levels in %s", fn);
        return JSC_ERR_TABLE;
      }
      tb->nt[np] = -1;
    }
    if (temp != temp_old || tb->nt[np] < 0) {
      temp_old = temp;
      if (++tb->nt[np] >= TBLNTMAX) {
        jsc_set_error(JSC_ERR_TABLE, "Too many temperatures in %s", fn);
        return JSC_ERR_TABLE;
      }
      tb->nu[np][tb->nt[np]] = -1;
    }
    int *nu = &tb->nu[np][tb->nt[np]];
    if ((eps > eps_old && u > u_old) || *nu < 0) {
      eps_old = eps;
      u_old = u;
      if (++(*nu) >= TBLNUMAX) {
        (*nu)--;
        continue;
      }
    }
    tb->p[np] = press;
    tb->t[np][tb->nt[np]] = temp;
    size_t row = ((size_t)np * TBLNTMAX + (size_t)tb->nt[np]) * RS;
    ubuf[row + (size_t)*nu] = (float)u;
    ebuf[row + (size_t)*nu] = (float)eps;
  }
  tb->np = np + 1;
  for (int ip = 0; ip < tb->np; ip++) {
    tb->nt[ip]++;
    for (int it = 0; it < tb->nt[ip]; it++) {
      int n = ++tb->nu[ip][it];
      int st = tables_reserve(ht, n);
      if (st) return st;
      size_t row = ((size_t)ip * TBLNTMAX + (size_t)it) * RS;
      tb->off[ip][it] = ht->n_points;
      memcpy(ht->u + ht->n_points, ubuf + row, (size_t)n * sizeof(float));
      memcpy(ht->eps + ht->n_points, ebuf + row, (size_t)n * sizeof(float));
      ht->n_points += n;
    }
  }
  return JSC_OK;
}

/* ---------------------------------------------- parallel binary loading */

/* A binary table file mapped into memory and walked with bounds checks. */
typedef struct {
  const unsigned char *data;
  size_t size, pos;
} bin_cursor;

static int cur_read(bin_cursor *c, void *dst, size_t bytes) {
  if (bytes > c->size - c->pos) return 0;
  if (dst) memcpy(dst, c->data + c->pos, bytes);
  c->pos += bytes;
  return 1;
}

/* Table header and row sizes of a mapped .bin file (the layout of
 * read_table_bin); returns its point count in *npts, or a JSC status with
 * the message in msg (set by the calling thread afterwards: the error
 * state is per thread). */
static int scan_table_bin(bin_cursor *c, jsc_host_table *tb, int64_t *npts, const char **msg) {
  int64_t n_all = 0;
  if (!cur_read(c, &tb->np, sizeof(int))) goto bad;
  if (tb->np > TBLNPMAX) {
    *msg = "Too many pressure levels";
    return JSC_ERR_TABLE;
  }
  if (tb->np < 0) tb->np = 0;
  if (!cur_read(c, tb->p, sizeof(double) * (size_t)tb->np)) goto bad;
  if (!cur_read(c, tb->nt, sizeof(int) * (size_t)tb->np)) goto bad;
  for (int ip = 0; ip < tb->np; ip++) {
    if (tb->nt[ip] > TBLNTMAX) {
      *msg = "Too many temperatures";
      return JSC_ERR_TABLE;
    }
    if (tb->nt[ip] < 0) tb->nt[ip] = 0;
    if (!cur_read(c, tb->t[ip], sizeof(double) * (size_t)tb->nt[ip])) goto bad;
    if (!cur_read(c, tb->nu[ip], sizeof(int) * (size_t)tb->nt[ip])) goto bad;
    for (int it = 0; it < tb->nt[ip]; it++) {
      int n = tb->nu[ip][it];
      if (n > TBLNUMAX) {
        *msg = "Too many column densities";
        return JSC_ERR_TABLE;
      }
      if (n < 0) n = tb->nu[ip][it] = 0;
      tb->off[ip][it] = (int64_t)c->pos;  /* file position of the row for now */
      if (!cur_read(c, NULL, 2 * sizeof(float) * (size_t)n)) goto bad;
      n_all += n;
    }
  }
  *npts = n_all;
  return JSC_OK;
bad:
  *msg = "Error while reading";
  return JSC_ERR_FILE;
}

/* All tables in binary form: the files are mapped and scanned in parallel,
 * placed back to back in table order (the layout of the serial reader),
 * and their rows copied in parallel.  Returns 1 in *fallback, without
 * touching ht, when a table is missing in binary form. */
static int read_tables_bin_parallel(const ctl_t *ctl, jsc_host_tables *ht, int *fallback) {
  const int nt = ctl->ng * ctl->nd;
  *fallback = 0;
  char (*names)[2 * LEN] = (char (*)[2 * LEN])malloc((size_t)(nt > 0 ? nt : 1) * 2 * LEN);
  bin_cursor *cur = (bin_cursor *)calloc((size_t)(nt > 0 ? nt : 1), sizeof(bin_cursor));
  int64_t *npts = (int64_t *)calloc((size_t)nt + 1, sizeof(int64_t));
  int *tst = (int *)calloc((size_t)(nt > 0 ? nt : 1), sizeof(int));
  const char **tmsg = (const char **)calloc((size_t)(nt > 0 ? nt : 1), sizeof(char *));
  int st = JSC_OK;
  if (!names || !cur || !npts || !tst || !tmsg) {
    st = JSC_ERR_NOMEM;
    goto out;
  }
  for (int i = 0; i < nt && !*fallback; i++) {
    const int id = i / ctl->ng, ig = i % ctl->ng;
    snprintf(names[i], 2 * LEN, "%s_%.4f_%s.bin", ctl->tblbase, ctl->nu[id], ctl->emitter[ig]);
    if (access(names[i], R_OK)) *fallback = 1;
  }
  if (*fallback) goto out;
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nt; i++) {
    const int fd = open(names[i], O_RDONLY);
    struct stat sb;
    if (fd < 0 || fstat(fd, &sb)) {
      tst[i] = JSC_ERR_FILE;
      tmsg[i] = "Error while reading";
      if (fd >= 0) close(fd);
      continue;
    }
    void *map = sb.st_size > 0 ? mmap(NULL, (size_t)sb.st_size, PROT_READ, MAP_PRIVATE, fd, 0)
                               : NULL;
    close(fd);
    if (sb.st_size > 0 && map == MAP_FAILED) {
      tst[i] = JSC_ERR_FILE;
      tmsg[i] = "Error while reading";
      continue;
    }
    cur[i].data = (const unsigned char *)map;
    cur[i].size = (size_t)sb.st_size;
    tst[i] = scan_table_bin(&cur[i], &ht->tab[i], &npts[i], &tmsg[i]);
  }
  for (int i = 0; i < nt; i++)
    if (tst[i]) {
      jsc_set_error(tst[i], "%s in %s", tmsg[i], names[i]);
      st = tst[i];
      goto out;
    }
  {
    int64_t total = 0;
    for (int i = 0; i < nt; i++) {
      const int64_t n = npts[i];
      npts[i] = total;  /* first point of table i */
      total += n;
    }
    if ((st = tables_reserve(ht, total + 1))) goto out;
    ht->n_points = total;
  }
#pragma omp parallel for schedule(dynamic)
  for (int i = 0; i < nt; i++) {
    jsc_host_table *tb = &ht->tab[i];
    int64_t o = npts[i];
    for (int ip = 0; ip < tb->np; ip++)
      for (int it = 0; it < tb->nt[ip]; it++) {
        const int n = tb->nu[ip][it];
        const unsigned char *row = cur[i].data + tb->off[ip][it];
        memcpy(ht->u + o, row, (size_t)n * sizeof(float));
        memcpy(ht->eps + o, row + (size_t)n * sizeof(float), (size_t)n * sizeof(float));
        tb->off[ip][it] = o;
        o += n;
      }
  }
out:
  if (cur)
    for (int i = 0; i < nt; i++)
      if (cur[i].data) munmap((void *)cur[i].data, cur[i].size);
  free(names);
  free(cur);
  free(npts);
  free(tst);
  free(tmsg);
  return st;
}

static int read_tables(const ctl_t *ctl, jsc_host_tables *ht) {
  char fn[2 * LEN];
  float *ubuf = NULL, *ebuf = NULL;
  int st = JSC_OK;
  ht->ng = ctl->ng;
  ht->nd = ctl->nd;
  ht->tab = (jsc_host_table *)calloc((size_t)(ctl->ng * ctl->nd + 1),
                                     sizeof(jsc_host_table));
  if (!ht->tab) return JSC_ERR_NOMEM;
  /* Every table in binary form: parallel mapped reads.  Otherwise (a .tab
   * or missing table) the serial reader below, file by file. */
  int fallback = 0;
  st = read_tables_bin_parallel(ctl, ht, &fallback);
  if (st || !fallback) return st;
  for (int id = 0; id < ctl->nd && !st; id++)
    for (int ig = 0; ig < ctl->ng && !st; ig++) {
      jsc_host_table *tb = &ht->tab[id * ctl->ng + ig];
      snprintf(fn, sizeof(fn), "%s_%.4f_%s.bin", ctl->tblbase, ctl->nu[id],
               ctl->emitter[ig]);
      FILE *in = fopen(fn, "r");
      if (in) {
        st = read_table_bin(in, fn, ht, tb);
        fclose(in);
        continue;
      }
      snprintf(fn, sizeof(fn), "%s_%.4f_%s.tab", ctl->tblbase, ctl->nu[id],
               ctl->emitter[ig]);
      in = fopen(fn, "r");
      if (!in) {
        /* Same outcome as the reference: a missing table contributes no
         * absorption (np < 2 gives eps = 0). */
        fprintf(stderr, "Missing emissivity table: %s\n", fn);
        tb->np = -1;
        continue;
      }
      if (!ubuf) {
        size_t nbuf = (size_t)TBLNPMAX * TBLNTMAX * TBLNUMAX;
        ubuf = (float *)malloc(nbuf * sizeof(float));
        ebuf = (float *)malloc(nbuf * sizeof(float));
        if (!ubuf || !ebuf) st = JSC_ERR_NOMEM;
      }
      if (!st) st = read_table_tab(in, fn, ht, tb, ubuf, ebuf);
      fclose(in);
    }
  free(ubuf);
  free(ebuf);
  return st;
}

/* ------------------------------------------------------------- filters */

/* Two-column shape file (src/forwardmodel.c:577-606). */
int jsc_read_filter(const char *filename, double *x, double *y, int *n) {
  char line[LEN];
  FILE *in = fopen(filename, "r");
  if (!in) {
    jsc_set_error(JSC_ERR_FILE, "Cannot open file %s", filename);
    return JSC_ERR_FILE;
  }
  *n = 0;
  while (fgets(line, LEN, in)) {
    double a, b;
    if (sscanf(line, "%lg %lg", &a, &b) == 2) {
      if (*n >= NSHAPE) {
        fclose(in);
        jsc_set_error(JSC_ERR_FILE, "Too many data points in %s", filename);
        return JSC_ERR_FILE;
      }
      x[*n] = a;
      y[*n] = b;
      (*n)++;
    }
  }
  fclose(in);
  if (*n < 1) {
    jsc_set_error(JSC_ERR_FILE, "Could not read any data from %s", filename);
    return JSC_ERR_FILE;
  }
  return JSC_OK;
}

double planck(double t, double nu) {
  return JSC_C1 * (nu * nu * nu) / jsc_gsl_expm1(JSC_C2 * nu / t);
}

/* Filter-weighted Planck table per channel (src/forwardmodel.c:757-786),
 * plus the slope of each interval in the form LIN evaluates it. */
static int planck_tables(const ctl_t *ctl, jsc_host_model *hm) {
  int st = JSC_OK;
  size_t n = (size_t)ctl->nd * JSC_NPLANCK;
  hm->planck_b = (double *)malloc(n * sizeof(double));
  hm->planck_s = (double *)malloc(n * sizeof(double));
  if (!hm->planck_b || !hm->planck_s) return JSC_ERR_NOMEM;
#pragma omp parallel for schedule(dynamic)
  for (int id = 0; id < ctl->nd; id++) {
    char fn[2 * LEN];
    double *fx = (double *)malloc(NSHAPE * sizeof(double));
    double *fy = (double *)malloc(NSHAPE * sizeof(double));
    int nf = 0, lst;
    snprintf(fn, sizeof(fn), "%s_%.4f.filt", ctl->tblbase, ctl->nu[id]);
    lst = (fx && fy) ? jsc_read_filter(fn, fx, fy, &nf) : JSC_ERR_NOMEM;
    if (lst) {
#pragma omp critical
      st = lst;
    } else {
      double *b = hm->planck_b + (size_t)id * JSC_NPLANCK;
      double *s = hm->planck_s + (size_t)id * JSC_NPLANCK;
      for (int it = 0; it < JSC_NPLANCK; it++) {
        double temp = jsc_lin(0.0, JSC_PLANCK_TMIN, JSC_NPLANCK - 1.0,
                              JSC_PLANCK_TMAX, (double)it);
        double fsum = 0, acc = 0;
        for (int i = 0; i < nf; i++) {
          fsum += fy[i];
          acc += fy[i] * planck(temp, fx[i]);
        }
        b[it] = acc / fsum;
      }
      for (int it = 0; it < JSC_NPLANCK; it++) {
        if (it + 1 < JSC_NPLANCK) {
          double t0 = jsc_lin(0.0, JSC_PLANCK_TMIN, JSC_NPLANCK - 1.0,
                              JSC_PLANCK_TMAX, (double)it);
          double t1 = jsc_lin(0.0, JSC_PLANCK_TMIN, JSC_NPLANCK - 1.0,
                              JSC_PLANCK_TMAX, (double)(it + 1));
          s[it] = (b[it + 1] - b[it]) / (t1 - t0);
        } else {
          s[it] = 0;
        }
      }
    }
    free(fx);
    free(fy);
  }
  if (st) jsc_set_error(st, "Cannot read filter functions below %s",
                        ctl->tblbase);
  return st;
}

/* ------------------------------------------------------------ continua */

/* Per-channel part of ctmco2/ctmh2o/ctmn2/ctmo2 (src/continua.c:5-2049):
 * the wavenumber interpolation of the coefficient tables and every factor
 * that depends on the channel only, each computed with the reference's
 * expression so the device finishes the same arithmetic per LOS point. */
void jsc_ctm_coefficients(const ctl_t *ctl, jsc_ctm_coef *c, int id) {
  double nu = ctl->nu[id];
  memset(c, 0, sizeof(*c));

  /* CO2 (src/continua.c:853-870) */
  double xw = nu / 2 + 1;
  if (xw >= 1 && xw < 2001) {
    int iw = (int)xw, jw = iw + 1;
    double dw = xw - iw, ew = 1 - dw;
    c->co2_on = 1;
    c->co2_c296 = ew * jsc_ckd_co2_t296[iw - 1] + dw * jsc_ckd_co2_t296[jw - 1];
    c->co2_c260 = ew * jsc_ckd_co2_t260[iw - 1] + dw * jsc_ckd_co2_t260[jw - 1];
    c->co2_c230 = ew * jsc_ckd_co2_t230[iw - 1] + dw * jsc_ckd_co2_t230[jw - 1];
  }

  /* H2O (src/continua.c:1901-1929) */
  xw = nu / 10 + 1;
  if (xw >= 1 && xw < 2001) {
    int iw = (int)xw, jw = iw + 1;
    double dw = xw - iw, ew = 1 - dw, sfac;
    double cw296 = ew * jsc_ckd_h2o_t296[iw - 1] + dw * jsc_ckd_h2o_t296[jw - 1];
    double cw260 = ew * jsc_ckd_h2o_t260[iw - 1] + dw * jsc_ckd_h2o_t260[jw - 1];
    double cwfrn = ew * jsc_ckd_h2o_frn[iw - 1] + dw * jsc_ckd_h2o_frn[jw - 1];
    if (nu <= 820 || nu >= 960) {
      sfac = 1;
    } else {
      double xx = (nu - 820) / 10;
      int ix = (int)xx;
      double dx = xx - ix;
      sfac = (1 - dx) * jsc_ckd_h2o_xfc[ix] + dx * jsc_ckd_h2o_xfc[ix + 1];
    }
    double vf2 = (nu - 370) * (nu - 370);
    double vf6 = vf2 * vf2 * vf2;
    double fscal = 36100 / (vf2 + vf6 * 1e-8 + 36100) * -.25 + 1;
    c->h2o_on = 1;
    c->h2o_self296 = sfac * cw296;
    c->h2o_ratio = cw260 / cw296;
    c->h2o_frn = cwfrn * fscal;
  }

  /* N2 (src/continua.c:1981-1988) */
  if (!(nu < jsc_n2_nu[0] || nu > jsc_n2_nu[97])) {
    int idx = jsc_locate(jsc_n2_nu, 98, nu);
    c->n2_on = 1;
    c->n2_b = jsc_lin(jsc_n2_nu[idx], jsc_n2_b[idx], jsc_n2_nu[idx + 1],
                      jsc_n2_b[idx + 1], nu);
    c->n2_beta = jsc_lin(jsc_n2_nu[idx], jsc_n2_beta[idx], jsc_n2_nu[idx + 1],
                         jsc_n2_beta[idx + 1], nu);
  }

  /* O2 (src/continua.c:2039-2045) */
  if (!(nu < jsc_o2_nu[0] || nu > jsc_o2_nu[89])) {
    int idx = jsc_locate(jsc_o2_nu, 90, nu);
    c->o2_on = 1;
    c->o2_b = jsc_lin(jsc_o2_nu[idx], jsc_o2_b[idx], jsc_o2_nu[idx + 1],
                      jsc_o2_b[idx + 1], nu);
    c->o2_beta = jsc_lin(jsc_o2_nu[idx], jsc_o2_beta[idx], jsc_o2_nu[idx + 1],
                         jsc_o2_beta[idx + 1], nu);
  }
}

/* --------------------------------------------------------------- model */

int jsc_host_model_load(const ctl_t *ctl, jsc_host_model *hm) {
  int st;
  memset(hm, 0, sizeof(*hm));
  if (ctl->ng < 0 || ctl->ng > NGMAX || ctl->nd < 1 || ctl->nd > NDMAX ||
      ctl->nw < 0 || ctl->nw > NWMAX) {
    jsc_set_error(JSC_ERR_ARG, "Invalid NG/ND/NW (%d/%d/%d)", ctl->ng,
                  ctl->nd, ctl->nw);
    return JSC_ERR_ARG;
  }
  hm->ng = ctl->ng;
  hm->nd = ctl->nd;
  hm->nw = ctl->nw;
  for (int id = 0; id < ctl->nd; id++) {
    hm->nu[id] = ctl->nu[id];
    hm->window[id] = ctl->window[id];
    if (ctl->window[id] < 0 || ctl->window[id] >= NWMAX) {
      jsc_set_error(JSC_ERR_ARG, "Invalid WINDOW[%d]=%d", id, ctl->window[id]);
      return JSC_ERR_ARG;
    }
  }
  hm->ig_co2 = jsc_find_emitter(ctl, "CO2");
  hm->ig_h2o = jsc_find_emitter(ctl, "H2O");
  hm->ctm_co2 = ctl->ctm_co2;
  hm->ctm_h2o = ctl->ctm_h2o;
  hm->ctm_n2 = ctl->ctm_n2;
  hm->ctm_o2 = ctl->ctm_o2;
  for (int id = 0; id < ctl->nd; id++) jsc_ctm_coefficients(ctl, &hm->ctm[id], id);
  if ((st = read_tables(ctl, &hm->tables))) return st;
  if ((st = planck_tables(ctl, hm))) return st;
  return JSC_OK;
}

/* The emissivity tables of ctl alone (read_tbl's part of the model). */
int jsc_read_tables(const ctl_t *ctl, jsc_host_tables *ht) {
  memset(ht, 0, sizeof(*ht));
  if (ctl->ng < 0 || ctl->ng > NGMAX || ctl->nd < 1 || ctl->nd > NDMAX) {
    jsc_set_error(JSC_ERR_ARG, "Invalid NG/ND (%d/%d)", ctl->ng, ctl->nd);
    return JSC_ERR_ARG;
  }
  return read_tables(ctl, ht);
}

/* The filter-weighted Planck tables of ctl's channels alone. */
int jsc_planck_only(const ctl_t *ctl, jsc_host_model *hm) {
  memset(hm, 0, sizeof(*hm));
  if (ctl->nd < 1 || ctl->nd > NDMAX) {
    jsc_set_error(JSC_ERR_ARG, "Invalid ND (%d)", ctl->nd);
    return JSC_ERR_ARG;
  }
  hm->nd = ctl->nd;
  return planck_tables(ctl, hm);
}

void jsc_host_model_free(jsc_host_model *hm) {
  free(hm->tables.tab);
  free(hm->tables.u);
  free(hm->tables.eps);
  free(hm->planck_b);
  free(hm->planck_s);
  memset(hm, 0, sizeof(*hm));
}
