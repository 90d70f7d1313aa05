/*
 * Aerosol/cloud optical properties: read_aero and get_opt_prop
 * (src/scatter.c:330-640) with the Mie evaluations on the GPU (mie.cu).
 *
 * The host part keeps the reference's bookkeeping: modes grouped into
 * layers by their top altitude, per mode either a log-normal Mie size
 * integral (opt_prop_mie_log, src/scatter.c:442-512) or the nearest record
 * of an external database (opt_prop_external, :516-580), and the layer sums
 * of extinction, scattering, absorption and phase function.  All Mie terms
 * of a call (modes x radius nodes x channels) go to the GPU in one launch;
 * the size integral then sums them in the reference's order (radius node,
 * then channel), so only the Mie series' own rounding differs.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "jsc_internal.h"

#define RAD_MIN 0.001   /* radius range of the size integral [micron] */
#define RAD_MAX 1000.

/* Gauss-Hermite abscissas (descending) and weights of NRAD nodes:
 * Newton iteration on the orthonormal Hermite recurrence with the
 * asymptotic starting values of Numerical Recipes (3rd ed., section 4.6),
 * the construction gauher (src/scatter.c:237-327) follows. */
static int gauss_hermite(double *z, double *w) {
  const int n = NRAD, half = (NRAD + 1) / 2;
  const double pim4 = 0.7511255444649425; /* pi^(-1/4) */
  double r = 0;
  for (int i = 0; i < half; i++) {
    if (i == 0)
      r = sqrt((double)(2 * n + 1)) - 1.85575 * pow((double)(2 * n + 1), -0.16667);
    else if (i == 1)
      r -= 1.14 * pow((double)n, 0.426) / r;
    else if (i == 2)
      r = 1.86 * r - 0.86 * z[0];
    else if (i == 3)
      r = 1.91 * r - 0.91 * z[1];
    else
      r = 2.0 * r - z[i - 2];
    double dp = 0;
    int it;
    for (it = 0; it < 10000; it++) {
      double h0 = pim4, h1 = 0.0;  /* H_j, H_{j-1} (orthonormal) */
      for (int j = 0; j < n; j++) {
        const double h2 = h1;
        h1 = h0;
        h0 = r * sqrt(2.0 / ((double)j + 1)) * h1 - sqrt((double)j / (j + 1.)) * h2;
      }
      dp = sqrt(2. * (double)n) * h1;  /* H_n' */
      const double r0 = r;
      r = r0 - h0 / dp;
      if (fabs(r - r0) <= 1.0e-14) break;
    }
    if (it >= 10000) {
      jsc_set_error(JSC_ERR_ARG, "Gauss-Hermite nodes did not converge");
      return JSC_ERR_ARG;
    }
    z[i] = r;
    z[n - 1 - i] = -r;
    w[i] = 2.0 / (dp * dp);
    w[n - 1 - i] = w[i];
  }
  return JSC_OK;
}

/* Next whitespace-separated token of a line (strtok on " \t"). */
static char *next_tok(char *line) { return strtok(line, " \t"); }

int jsc_read_aero(const char *dirname, const char *filename, const ctl_t *ctl, aero_t *aero) {
  char file[2 * LEN + 2], *line = (char *)malloc(LEN);
  if (!line) return JSC_ERR_NOMEM;
  if (dirname)
    snprintf(file, sizeof(file), "%s/%s", dirname, filename);
  else
    snprintf(file, sizeof(file), "%s", filename);
  FILE *in = fopen(file, "r");
  if (!in) {
    free(line);
    jsc_set_error(JSC_ERR_FILE, "cannot open aerosol file %s", file);
    return JSC_ERR_FILE;
  }
  aero->nm = 0;
  int st = JSC_OK;
  while (!st && fgets(line, LEN, in)) {
    const int im = aero->nm;
    char *tok;
    double v[6];
    char type[LEN], path[LEN];
    int ok = 1;
    /* top bottom trans type file nn rr ss, as read_aero's TOK sequence:
     * a missing token is an error, an unparsable one skips the line */
    for (int f = 0; f < 8 && ok; f++) {
      tok = next_tok(f == 0 ? line : NULL);
      if (!tok) {
        jsc_set_error(JSC_ERR_FILE, "error while reading %s", file);
        st = JSC_ERR_FILE;
        ok = 0;
        break;
      }
      if (f == 3 || f == 4) {
        if (sscanf(tok, "%s", f == 3 ? type : path) != 1) ok = 0;
      } else if (sscanf(tok, "%lg", &v[f < 3 ? f : f - 2]) != 1) {
        ok = 0;
      }
    }
    if (st || !ok) continue;
    if (im >= SCAMOD) {
      jsc_set_error(JSC_ERR_ARG, "too many aerosol models in %s", file);
      st = JSC_ERR_ARG;
      break;
    }
    aero->top_mod[im] = v[0];
    aero->bottom_mod[im] = v[1];
    aero->trans_mod[im] = v[2];
    snprintf(aero->type[im], LEN, "%s", type);
    snprintf(aero->filepath[im], LEN, "%s", path);
    aero->nn[im] = v[3];
    aero->rr[im] = v[4];
    aero->ss[im] = v[5];
    aero->nm++;
  }
  fclose(in);
  free(line);
  if (st) return st;
  if (aero->nm < 1) {
    jsc_set_error(JSC_ERR_FILE, "could not read any aerosol data from %s", file);
    return JSC_ERR_FILE;
  }
  if (ctl->sca_n != aero->nm) {
    jsc_set_error(JSC_ERR_ARG, "SCA_N=%d but %d aerosol models in %s", ctl->sca_n, aero->nm,
                  file);
    return JSC_ERR_ARG;
  }
  return JSC_OK;
}

/* Refractive index of a Mie mode at every channel: the file's (nu, n, k)
 * records interpolated linearly (src/scatter.c:460-482). */
static int refractive_index(const ctl_t *ctl, const char *path, double *nr, double *ni) {
  FILE *in = fopen(path, "r");
  if (!in) {
    jsc_set_error(JSC_ERR_FILE, "cannot open refractive-index file %s", path);
    return JSC_ERR_FILE;
  }
  double *nu = (double *)malloc(3 * (REFMAX + 1) * sizeof(double));
  char *line = (char *)malloc(LEN);
  if (!nu || !line) {
    fclose(in);
    free(nu);
    free(line);
    return JSC_ERR_NOMEM;
  }
  double *rn = nu + REFMAX + 1, *rk = rn + REFMAX + 1;
  int np = 0, st = JSC_OK;
  while (fgets(line, LEN, in))
    if (sscanf(line, "%lg %lg %lg", &nu[np], &rn[np], &rk[np]) == 3)
      if (++np > REFMAX) {
        jsc_set_error(JSC_ERR_ARG, "too many refractive-index records in %s", path);
        st = JSC_ERR_ARG;
        break;
      }
  fclose(in);
  if (!st && np < 2) {
    jsc_set_error(JSC_ERR_FILE, "fewer than two refractive-index records in %s", path);
    st = JSC_ERR_FILE;
  }
  if (!st)
    for (int id = 0; id < ctl->nd; id++) {
      const int i = jsc_locate(nu, np, ctl->nu[id]);
      nr[id] = jsc_lin(nu[i], rn[i], nu[i + 1], rn[i + 1], ctl->nu[id]);
      ni[id] = jsc_lin(nu[i], rk[i], nu[i + 1], rk[i + 1], ctl->nu[id]);
    }
  free(nu);
  free(line);
  return st;
}

/* External database mode (opt_prop_external, src/scatter.c:516-580): the
 * record of the nearest wavenumber per channel. */
static int external_mode(const ctl_t *ctl, const aero_t *aero, int im, double *be, double *bs,
                         double *ph) {
  if (aero->nn[im] == 1) {
    jsc_set_error(JSC_ERR_UNSUPPORTED, "interpolated external optical properties (nn = 1)");
    return JSC_ERR_UNSUPPORTED;
  }
  if (aero->nn[im] != 0) return JSC_OK;  /* the reference sets nothing */
  FILE *in = fopen(aero->filepath[im], "r");
  if (!in) {
    jsc_set_error(JSC_ERR_FILE, "cannot open optical-property file %s", aero->filepath[im]);
    return JSC_ERR_FILE;
  }
  const size_t rec = 3 + NTHETA;
  double *db = (double *)malloc((size_t)(REFMAX + 1) * rec * sizeof(double));
  char *line = (char *)malloc(LEN);
  double *nu = (double *)malloc((REFMAX + 1) * sizeof(double));
  int np = 0, st = JSC_OK;
  if (!db || !line || !nu) st = JSC_ERR_NOMEM;
  while (!st && fgets(line, LEN, in)) {
    double *r = db + (size_t)np * rec;
    int ok = 1;
    for (size_t f = 0; f < rec && ok; f++) {
      char *tok = next_tok(f == 0 ? line : NULL);
      if (!tok) {
        jsc_set_error(JSC_ERR_FILE, "error while reading %s", aero->filepath[im]);
        st = JSC_ERR_FILE;
        ok = 0;
      } else if (sscanf(tok, "%lg", &r[f]) != 1) {
        ok = 0;
      }
    }
    if (st || !ok) continue;
    nu[np] = r[0];
    if (++np > REFMAX) {
      jsc_set_error(JSC_ERR_ARG, "too many records in %s", aero->filepath[im]);
      st = JSC_ERR_ARG;
    }
  }
  fclose(in);
  if (!st && np < 1) {
    jsc_set_error(JSC_ERR_FILE, "could not read any data from %s", aero->filepath[im]);
    st = JSC_ERR_FILE;
  }
  if (!st)
    for (int id = 0; id < ctl->nd; id++) {
      int i = jsc_locate(nu, np, ctl->nu[id]);
      if (np >= 2 && fabs(nu[i] - ctl->nu[id]) > fabs(nu[i + 1] - ctl->nu[id])) i++;
      const double *r = db + (size_t)i * rec;
      be[id] = r[1];
      bs[id] = r[2];
      for (int it = 0; it < NTHETA; it++) ph[(size_t)id * NTHETA + it] = r[3 + it];
    }
  free(db);
  free(line);
  free(nu);
  return st;
}

static int gpu_device(void) {
  const char *s = getenv("JURASSIC_GPU_DEVICE");
  return s ? atoi(s) : 0;
}

int jsc_get_opt_prop(const ctl_t *ctl, aero_t *aero) {
  const int nd = ctl->nd, nm = aero->nm;
  if (nd < 1 || nd > NDMAX || nm < 1 || nm > SCAMOD) {
    jsc_set_error(JSC_ERR_ARG, "jsc_get_opt_prop: invalid sizes (nd=%d nm=%d)", nd, nm);
    return JSC_ERR_ARG;
  }
  /* Layers from the modes' top altitudes (src/scatter.c:334-372). */
  if (aero->top_mod[0] <= aero->bottom_mod[0]) {
    jsc_set_error(JSC_ERR_ARG, "aerosol top altitude is not above the bottom altitude");
    return JSC_ERR_ARG;
  }
  int nl = 1, cnt = 1;
  aero->top[0] = aero->top_mod[0];
  aero->bottom[0] = aero->bottom_mod[0];
  aero->trans[0] = aero->trans_mod[0];
  for (int im = 1; im < nm; im++) {
    if (aero->top_mod[im] > aero->top_mod[im - 1] || aero->top_mod[im] <= aero->bottom_mod[im] ||
        aero->bottom_mod[im] > aero->bottom_mod[im - 1]) {
      jsc_set_error(JSC_ERR_ARG, "aerosol/cloud altitudes or transition layers are wrong");
      return JSC_ERR_ARG;
    }
    if (aero->top_mod[im] != aero->top_mod[im - 1]) {
      if (nl >= NLMAX) {
        jsc_set_error(JSC_ERR_ARG, "more than %d aerosol/cloud layers", NLMAX);
        return JSC_ERR_ARG;
      }
      aero->top[nl] = aero->top_mod[im];
      aero->bottom[nl] = aero->bottom_mod[im];
      aero->trans[nl] = aero->trans_mod[im];
      aero->nmod[nl - 1] = cnt;
      nl++;
      cnt = 0;
    }
    cnt++;
  }
  aero->nmod[nl - 1] = cnt;
  aero->nl = nl;

  /* Mie tasks of every MIE mode: valid radius nodes x channels. */
  double zs[NRAD], ws[NRAD];
  int st = gauss_hermite(zs, ws);
  if (st) return st;
  int ntask = 0;
  for (int im = 0; im < nm; im++) {
    if (strcasecmp(aero->type[im], "MIE")) continue;
    if (aero->nn[im] <= 0 || aero->rr[im] <= 0 || aero->ss[im] <= 1) {
      jsc_set_error(JSC_ERR_ARG, "log-normal parameters of mode %d are not physical", im);
      return JSC_ERR_ARG;
    }
    ntask += NRAD * nd;
  }
  double *tx = (double *)malloc(((size_t)ntask * 3 + 1) * sizeof(double));
  double *out = (double *)malloc(((size_t)ntask * (2 + NTHETA) + 1) * sizeof(double));
  double *mode = (double *)malloc((size_t)nd * (2 + NTHETA) * sizeof(double));
  double *nr = (double *)malloc(2 * (size_t)nd * sizeof(double));
  int *tid = (int *)malloc(((size_t)nm * NRAD * nd + 1) * sizeof(int));
  if (!tx || !out || !mode || !nr || !tid) {
    st = JSC_ERR_NOMEM;
    goto done;
  }
  {
    double *ni = nr + nd;
    int nt = 0;
    for (int im = 0; im < nm; im++) {
      if (strcasecmp(aero->type[im], "MIE")) continue;
      if ((st = refractive_index(ctl, aero->filepath[im], nr, ni))) goto done;
      const double k1 = aero->nn[im] * 1e-3 * sqrt(M_PI);
      for (int n = 0; n < NRAD; n++) {
        const double rad = exp(sqrt(2) * log(aero->ss[im]) * zs[n] + log(aero->rr[im]));
        for (int id = 0; id < nd; id++) {
          int *slot = &tid[((size_t)im * NRAD + n) * nd + id];
          *slot = -1;
          if (!(rad >= RAD_MIN && rad <= RAD_MAX && k1 > 0.)) continue;
          const double lambda = 1. / (ctl->nu[id]) * pow(10, 4.);
          tx[nt] = 2 * M_PI * rad / lambda;
          tx[ntask + nt] = nr[id];
          tx[2 * (size_t)ntask + nt] = ni[id];
          *slot = nt++;
        }
      }
    }
    if (nt > 0) {
      /* compact the refractive indices behind the nt size parameters */
      memmove(tx + nt, tx + ntask, nt * sizeof(double));
      memmove(tx + 2 * (size_t)nt, tx + 2 * (size_t)ntask, nt * sizeof(double));
      if ((st = jsc_mie_eval(gpu_device(), nt, tx, tx + nt, tx + 2 * (size_t)nt, out))) goto done;
    }

    /* Per layer: sum of its modes (src/scatter.c:374-430). */
    int im = 0;
    for (int il = 0; il < nl; il++) {
      for (int id = 0; id < nd; id++) {
        aero->beta_e[il][id] = aero->beta_s[il][id] = aero->beta_a[il][id] = 0.;
        for (int it = 0; it < NTHETA; it++) aero->p[il][id][it] = 0.;
      }
      for (int jm = 0; jm < aero->nmod[il]; jm++, im++) {
        double *be = mode, *bs = mode + nd, *ph = mode + 2 * nd;
        memset(mode, 0, (size_t)nd * (2 + NTHETA) * sizeof(double));
        if (!strcasecmp(aero->type[im], "MIE")) {
          /* size integral in the order of opt_prop_mie_log: radius node,
           * then channel */
          const double k1 = aero->nn[im] * 1e-3 * sqrt(M_PI);
          for (int n = 0; n < NRAD; n++) {
            const double rad = exp(sqrt(2) * log(aero->ss[im]) * zs[n] + log(aero->rr[im]));
            for (int id = 0; id < nd; id++) {
              const int t = tid[((size_t)im * NRAD + n) * nd + id];
              if (t < 0) continue;
              const double *o = out + (size_t)t * (2 + NTHETA);
              be[id] += k1 * pow(rad, 2) * o[0] * ws[n];
              bs[id] += k1 * pow(rad, 2) * o[1] * ws[n];
              for (int it = 0; it < NTHETA; it++)
                ph[(size_t)id * NTHETA + it] += k1 * o[1] * pow(rad, 2) * o[2 + it] * ws[n];
            }
          }
          for (int id = 0; id < nd; id++)
            for (int it = 0; it < NTHETA; it++) ph[(size_t)id * NTHETA + it] /= bs[id];
        } else if (!strcasecmp(aero->type[im], "Ext")) {
          if ((st = external_mode(ctl, aero, im, be, bs, ph))) goto done;
        } else if (!strcasecmp(aero->type[im], "Const")) {
          jsc_set_error(JSC_ERR_UNSUPPORTED, "constant-extinction aerosol model");
          st = JSC_ERR_UNSUPPORTED;
          goto done;
        } else {
          jsc_set_error(JSC_ERR_ARG, "unknown scattering model '%s' (MIE, Ext, Const)",
                        aero->type[im]);
          st = JSC_ERR_ARG;
          goto done;
        }
        for (int id = 0; id < nd; id++) {
          aero->beta_e[il][id] += be[id];
          aero->beta_s[il][id] += bs[id];
          aero->beta_a[il][id] += (be[id] - bs[id]);
          for (int it = 0; it < NTHETA; it++) aero->p[il][id][it] += ph[(size_t)id * NTHETA + it];
        }
      }
    }
  }
done:
  free(tx);
  free(out);
  free(mode);
  free(nr);
  free(tid);
  return st;
}
