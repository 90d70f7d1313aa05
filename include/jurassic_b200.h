/*
 * jurassic_b200.h -- public C interface of the B200 forward model.
 *
 * Two layers are declared here.
 *
 * 1. The drop-in layer.  formod(), brightness() and planck() keep the exact
 *    signatures of the reference forward model (src/forwardmodel.h:16-19,
 *    :282-283, :339-340), and the structs below keep the reference's memory
 *    layout (src/jurassic.h:228-570) field for field, so a program built
 *    against the reference headers links this library in place of
 *    forwardmodel.o.  Field names are the reference's because callers use
 *    them; sizes and offsets are checked by the test suite.
 *
 * 2. The plain C-ABI (jsc_*).  Opaque handles, plain pointers and sizes, no
 *    C++ or torch types.  formod() is a thin client of it; batch callers
 *    (many atmospheres and rays in one launch) call it directly.
 */
#ifndef JURASSIC_B200_H
#define JURASSIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Dimensions.  They size the fixed arrays of the boundary structs and must
 * equal the reference's compile-time values (src/jurassic.h:135-196).
 * ------------------------------------------------------------------------ */
#define LEN      5000   /* characters per text field */
#define NWMAX    5      /* spectral windows */
#define NDMAX    130    /* radiance channels */
#define NGMAX    25     /* emitters */
#define NLOS     10000  /* points per line of sight */
#define NPMAX    1000   /* atmospheric data points */
#define NRMAX    1000   /* ray paths per obs_t */
#define NSHAPE   10000  /* points of a filter or field-of-view shape */
#define NFOV     50     /* rays used for the field-of-view convolution */
#define TBLNPMAX 50     /* pressure levels per emissivity table */
#define TBLNSMAX 1201   /* temperatures of the Planck source table */
#define TBLNTMAX 30     /* temperatures per pressure level */
#define TBLNUMAX 320    /* column densities per (pressure, temperature) */
#define SCAMOD   30     /* aerosol/cloud models */
#define NLMAX    10     /* aerosol/cloud layers */
#define NTHETA   181    /* phase-function angles, 0..180 deg */
#define NRAD     170    /* Gauss-Hermite nodes of the size integral */
#define REFMAX   5000   /* refractive-index records */

/* Physical constants with the reference's values (src/jurassic.h:113-126;
 * GSL 1.15 gsl_const_mksa.h / gsl_const_num.h for the last three). */
#define JSC_C1        1.19104259e-8   /* 2hc^2 [W/(m^2 sr cm^-4)] */
#define JSC_C2        1.43877506      /* hc/k  [K/cm^-1] */
#define JSC_P0        1013.25         /* standard pressure [hPa] */
#define JSC_RE        6367.421        /* mean Earth radius [km] */
#define JSC_TSUN      5780.           /* solar temperature [K] */
#define JSC_KBOLTZ    1.3806504e-23   /* Boltzmann constant [J/K] */
#define JSC_RGAS      8.314472        /* molar gas constant [J/(mol K)] */
#define JSC_AVOGADRO  6.02214199e23   /* [1/mol] */

/* ------------------------------------------------------------------------
 * Boundary structs (layout of src/jurassic.h:13-25 and :228-570).
 * ------------------------------------------------------------------------ */

/* Work-queue bookkeeping carried inside ctl_t (src/workqueue.h:13-25).  The
 * GPU path keeps its own device-resident queue; these fields are only kept
 * for layout compatibility and are not touched by formod(). */
typedef struct {
  void *input;
  void *result;
  int ir;
} queue_item_t;

typedef struct {
  queue_item_t *items;
  int capacity;
  int begin;
  int end;
  int state;
} queue_t;

/* Forward-model control parameters, as filled by the reference's read_ctl. */
typedef struct {
  int ng;                       /* emitters */
  char emitter[NGMAX][LEN];     /* emitter names (table file suffixes) */
  int nd;                       /* channels */
  int nw;                       /* spectral windows */
  double nu[NDMAX];             /* channel centre wavenumbers [cm^-1] */
  int window[NDMAX];            /* window index of each channel */
  char tblbase[LEN];            /* base name of table and filter files */
  double hydz;                  /* hydrostatic reference height, <0: off [km] */
  int ctm_co2, ctm_h2o, ctm_n2, ctm_o2;   /* continua switches */
  int sca_n;                    /* aerosol/cloud models */
  int sca_mult;                 /* scattering depth: 0 none, 1 single, >=2 multiple */
  char sca_ext[LEN];            /* "beta_a" or "beta_e" when sca_mult==0 */
  int ip;                       /* atmosphere interpolation: 1 profile, 2, 3 */
  double cz, cx;                /* influence lengths for ip 2/3 [km] */
  int refrac;                   /* refraction on/off */
  double rayds;                 /* maximum ray step [km] */
  double raydz;                 /* vertical ray step [km] */
  double transs;                /* transition-layer sampling step [km] */
  char fov[LEN];                /* field-of-view file, "-" for none */
  double retp_zmin, retp_zmax;
  double rett_zmin, rett_zmax;
  double retq_zmin[NGMAX], retq_zmax[NGMAX];
  double retk_zmin[NWMAX], retk_zmax[NWMAX];
  double retnn_zmin, retnn_zmax;
  int retnn, retrr, retss;      /* aerosol retrieval switches */
  int write_bbt;                /* convert output to brightness temperature */
  int write_matrix;
  queue_t queue;
} ctl_t;

/* Observation geometry and results for up to NRMAX rays. */
typedef struct {
  int nr;
  double time[NRMAX];
  double obsz[NRMAX], obslon[NRMAX], obslat[NRMAX];
  double vpz[NRMAX], vplon[NRMAX], vplat[NRMAX];
  double tpz[NRMAX], tplon[NRMAX], tplat[NRMAX];
  double tau[NDMAX][NRMAX];     /* path transmittance */
  double rad[NDMAX][NRMAX];     /* radiance [W/(m^2 sr cm^-1)]; NaN = masked */
} obs_t;

/* Aerosol/cloud models and the optical properties derived from them. */
typedef struct {
  int nm;
  double top_mod[SCAMOD], bottom_mod[SCAMOD], trans_mod[SCAMOD];
  char type[SCAMOD][LEN];
  char filepath[SCAMOD][LEN];
  double nn[SCAMOD], rr[SCAMOD], ss[SCAMOD];
  int nl;
  int nmod[NLMAX];
  double top[NLMAX], bottom[NLMAX], trans[NLMAX];
  double beta_e[NLMAX][NDMAX];  /* extinction [1/km] */
  double beta_s[NLMAX][NDMAX];  /* scattering [1/km] */
  double beta_a[NLMAX][NDMAX];  /* absorption [1/km] */
  double p[NLMAX][NDMAX][NTHETA];  /* phase function */
} aero_t;

/* Atmospheric state (one or more profiles). */
typedef struct {
  int np;
  double time[NPMAX];
  double z[NPMAX], lon[NPMAX], lat[NPMAX];
  double p[NPMAX], t[NPMAX];
  double q[NGMAX][NPMAX];
  double k[NWMAX][NPMAX];
  int init;
} atm_t;

/* Line of sight of one ray (src/jurassic.h:352-393): what raytrace
 * writes and formod_pencil integrates.  Only the host helpers
 * formod_continua and intpol_tbl below take it; the GPU path keeps its own
 * packed LOS records in device memory. */
typedef struct {
  int np;
  double z[NLOS], lon[NLOS], lat[NLOS];
  double p[NLOS], t[NLOS];
  double q[NLOS][NGMAX];
  double k[NLOS][NWMAX];
  int aeroi[NLOS];              /* aerosol/cloud layer index */
  double aerofac[NLOS];         /* aerosol/cloud layer factor */
  double tsurf;                 /* surface temperature [K], <= 0: none */
  double ds[NLOS];              /* segment length [km] */
  double u[NLOS][NGMAX];        /* column density [molecules/cm^2] */
} los_t;

/* Emissivity look-up tables in the reference's fixed layout
 * (src/jurassic.h:438-471, about 12.5 GB): what read_tbl fills and the
 * host helpers intpol_tbl* read.  The GPU path never uses it; its device
 * tables hold only the rows that exist (jsc_model_create). */
typedef struct {
  int np[NGMAX][NDMAX];
  int nt[NGMAX][NDMAX][TBLNPMAX];
  int nu[NGMAX][NDMAX][TBLNPMAX][TBLNTMAX];
  double p[NGMAX][NDMAX][TBLNPMAX];
  double t[NGMAX][NDMAX][TBLNPMAX][TBLNTMAX];
  float u[NGMAX][NDMAX][TBLNPMAX][TBLNTMAX][TBLNUMAX];
  float eps[NGMAX][NDMAX][TBLNPMAX][TBLNTMAX][TBLNUMAX];
  double st[TBLNSMAX];
  double sr[NDMAX][TBLNSMAX];
} tbl_t;

/* ------------------------------------------------------------------------
 * Drop-in entry points.
 * ------------------------------------------------------------------------ */

/* Replaces formod (src/forwardmodel.c:15-116), for ctl->ip 1 (one
 * profile), 2 (profiles split where lon/lat change, the two nearest
 * blended) and 3 (points weighted within ctl->cz, cx; with scattering the
 * 3-D source of 32,400 secondary pencils per scattering point):
 * saves the NaN mask of
 * obs->rad, applies hydrostatic balance to atm->p (ctl->hydz >= 0), traces
 * every ray, evaluates EGA transmittances, continua, Planck source and
 * radiative transfer on the GPU (single/multiple scattering when
 * ctl->sca_mult > 0 and ctl->sca_n > 0), convolves with the field-of-view
 * shape of ctl->fov unless it is "-" (formod_fov, src/forwardmodel.c:
 * 156-220), converts to brightness temperature when ctl->write_bbt, and
 * restores the mask.  Writes obs->rad, obs->tau and
 * obs->tpz/tplon/tplat.  Errors follow the reference's ERRMSG convention
 * (message, exit(EXIT_FAILURE)) unless jsc_set_exit_on_error(0). */
void formod(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero);

/* Brightness temperature of a radiance (src/forwardmodel.c:7-11). */
double brightness(double rad, double nu);

/* Planck function (src/forwardmodel.c:569-573). */
double planck(double t, double nu);

/* The rest of the reference's forwardmodel.h (src/forwardmodel.h:21-85),
 * so that programs and objects written against it (its scatter.o calls
 * formod_pencil, misc.o read_shape) link this library in place of
 * forwardmodel.o.  Errors follow formod()'s convention. */

/* Replaces formod_pencil (src/forwardmodel.c:224-405): ray ir of obs
 * through atm as given (no hydrostatic balance, mask or field of view),
 * traced, refined at aerosol/cloud layer edges and integrated ON THE GPU
 * with scattering sources of order `scattering` (0: none, aerosol/cloud
 * extinction per ctl->sca_ext when ctl->sca_n > 0); writes obs->rad[*][ir],
 * obs->tau[*][ir] and obs->tpz/tplon/tplat[ir]. */
void formod_pencil(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, int scattering, int ir);

/* The scattering source of srcfunc_sca (src/scatter.c:643-662) at n points
 * at once, ON THE GPU: point k at Cartesian position x[3k..3k+2] [km] on a
 * line of sight along dx[3k..3k+2], in aerosol/cloud layer layer[k], at time
 * sec[k] [s since 2000-01-01T00:00Z]; the thermal source of the secondary
 * pencils of order scattering - 1 (srcfunc_sca_1d for ctl->ip 1,
 * srcfunc_sca_3d's 32,400 pencils for ip 2/3) plus the solar term
 * (srcfunc_sca_sun), into src[n][nd].  atm is taken as given (formod
 * applies the hydrostatic balance before its pencils call srcfunc_sca);
 * aero holds the layers and optical properties; ctl->sca_n must be > 0 and
 * scattering >= 1.  Returns a JSC_* status (no exit). */
int jsc_srcfunc_sca(ctl_t *ctl, atm_t *atm, aero_t *aero, int n, const double *x,
                    const double *dx, const int *layer, const double *sec, int scattering,
                    double *src);

/* Replaces formod_fov (src/forwardmodel.c:156-220): field-of-view
 * convolution of obs over tangent height with the shape of ctl->fov
 * (nothing when it is "-"); host post-processing, as in formod(). */
void formod_fov(ctl_t *ctl, obs_t *obs);

/* Replaces read_shape (src/forwardmodel.c:577-606): the two columns of a
 * filter or field-of-view file into x, y (NSHAPE points at most), *n the
 * count.  Host file input. */
void read_shape(const char *filename, double *x, double *y, int *n);

/* Host helpers on the reference's host-side structs (a caller's tbl_t and
 * los_t live in host memory; the GPU forward model never calls these).
 *
 * read_tbl (src/forwardmodel.c:610-739): the emissivity tables
 * <tblbase>_<nu>_<emitter>.bin, else .tab, of every (emitter, channel)
 * into tbl (np = -1 for a missing table); binary rows longer than
 * TBLNUMAX are refused rather than read misaligned.
 * srcfunc_planck (src/forwardmodel.c:743-794): filter-weighted Planck
 * source of every channel at temperature t into src[nd] (the table of a
 * channel set is built on first use and kept).
 * formod_continua (src/forwardmodel.c:120-152): continuum extinction of
 * every channel at LOS point ip into beta[nd].
 * intpol_tbl (src/forwardmodel.c:409-502): EGA transmittances of LOS point
 * ip; tau_path carries the path state (initialised to 1 at ip <= 0),
 * tau_seg[nd] receives the segment transmittance.
 * intpol_tbl_eps / intpol_tbl_u (src/forwardmodel.c:506-542): emissivity
 * at column density u, column density at emissivity eps, on row
 * (ig, id, ip, it).  locate_tbl (src/forwardmodel.c:546-565): bisection
 * on a float array, the largest i < n-1 with xx[i] <= x. */
void read_tbl(ctl_t *ctl, tbl_t *tbl);
void srcfunc_planck(ctl_t *ctl, double t, double *src);
void formod_continua(ctl_t *ctl, los_t *los, int ip, double *beta);
void intpol_tbl(ctl_t *ctl, tbl_t *tbl, los_t *los, int ip, double tau_path[NGMAX][NDMAX],
                double tau_seg[NDMAX]);
double intpol_tbl_eps(tbl_t *tbl, int ig, int id, int ip, int it, double u);
double intpol_tbl_u(tbl_t *tbl, int ig, int id, int ip, int it, double eps);
int locate_tbl(float *xx, int n, double x);

/* ------------------------------------------------------------------------
 * Plain C-ABI.
 * ------------------------------------------------------------------------ */

/* Status codes returned by every jsc_* call. */
enum {
  JSC_OK = 0,
  JSC_ERR_ARG = 1,        /* invalid argument or size */
  JSC_ERR_CUDA = 2,       /* CUDA runtime error */
  JSC_ERR_FILE = 3,       /* missing or unreadable input file */
  JSC_ERR_TABLE = 4,      /* emissivity table exceeds a dimension */
  JSC_ERR_NLOS = 5,       /* a ray needs more than NLOS points */
  JSC_ERR_OBSERVER = 6,   /* observer below the surface */
  JSC_ERR_QUEUE = 7,      /* scattering work queue over capacity */
  JSC_ERR_WATCHDOG = 8,   /* a device-side wait gave up */
  JSC_ERR_UNSUPPORTED = 9,/* feature outside the GPU path (ip != 1, FOV) */
  JSC_ERR_NOMEM = 10      /* host or device allocation failed */
};

/* Message of a status code. */
const char *jsc_status_string(int status);

/* Status of the last formod() call on this thread. */
int jsc_last_status(void);

/* formod() error behaviour: 1 (default) prints and exits like the
 * reference's ERRMSG, 0 returns with jsc_last_status() set. */
void jsc_set_exit_on_error(int on);

/* Message describing the last error on this thread. */
const char *jsc_last_error_message(void);

/* Release the model and batches that formod() and jsc_kernel() cache
 * between calls. */
void jsc_release_cache(void);

/* ------------------------------------------------------------------------
 * Aerosol/cloud optical properties.
 * ------------------------------------------------------------------------ */

/* Replaces read_aero (src/scatter.c:584-640): the modes of an aerosol
 * file (top, bottom, transition [km], type MIE/Ext/Const, property file,
 * and nn [cm^-3], rr [micron], ss for log-normal Mie modes) into
 * aero->nm and the *_mod / type / filepath / nn / rr / ss fields; the count
 * must equal ctl->sca_n.  dirname may be NULL. */
int jsc_read_aero(const char *dirname, const char *filename, const ctl_t *ctl, aero_t *aero);

/* Replaces get_opt_prop (src/scatter.c:330-437): groups the modes into
 * layers (aero->nl, nmod, top, bottom, trans) and fills beta_e, beta_s,
 * beta_a and the phase function p per layer and channel.  MIE modes
 * integrate the Bohren-Huffman Mie series over a log-normal size
 * distribution with 170 Gauss-Hermite radius nodes (opt_prop_mie_log); all
 * Mie series of the call run on the GPU in one launch, the size integral
 * sums them in the reference's order.  Ext modes take the nearest-
 * wavenumber record of their database file (opt_prop_external).  The GPU
 * is JURASSIC_GPU_DEVICE (default 0). */
int jsc_get_opt_prop(const ctl_t *ctl, aero_t *aero);

/* ------------------------------------------------------------------------
 * Jacobians (the retrieval's caller of the forward model).
 * ------------------------------------------------------------------------ */

/* Quantity codes of state-vector elements (IDXP..IDXSS, src/jurassic.h:
 * 203-221). */
#define JSC_IDXP 0
#define JSC_IDXT 1
#define JSC_IDXQ(ig) (2 + (ig))
#define JSC_IDXK(ctl, iw) (2 + (ctl)->ng + (iw))
#define JSC_IDXNN(ctl) (2 + (ctl)->ng + (ctl)->nw + 1)
#define JSC_IDXRR(ctl) (2 + (ctl)->ng + (ctl)->nw + 2)
#define JSC_IDXSS(ctl) (2 + (ctl)->ng + (ctl)->nw + 3)

/* State vector of atm and aero (atm2x, src/atmosphere.c:5-97): pressure,
 * temperature, volume mixing ratios and extinction at the levels inside
 * each quantity's ctl->ret*_zmin..zmax, then the aerosol parameters
 * selected by ctl->retnn/retrr/retss.  x, iqa (quantity codes) and ipa
 * (level, -1 for aerosol parameters) may be NULL.  Returns the length. */
size_t jsc_atm2x(const ctl_t *ctl, const atm_t *atm, const aero_t *aero, double *x,
                 int *iqa, int *ipa);

/* Inverse of jsc_atm2x (x2atm, src/retrievalmodel.c:1103-1163). */
void jsc_x2atm(const ctl_t *ctl, const double *x, atm_t *atm, aero_t *aero);

/* Measurement vector: the finite entries of obs->rad, ray-major
 * (obs2y, src/retrievalmodel.c:379-403).  y, ida, ira may be NULL.
 * Returns the length. */
size_t jsc_obs2y(const ctl_t *ctl, const obs_t *obs, double *y, int *ida, int *ira);

/* Replaces kernel (src/retrievalmodel.c:201-298): the Jacobian
 * k[i * tda + j] = (y_j[i] - y[i]) / h_j of the measurement vector with
 * respect to the state vector, by finite differences with the reference's
 * perturbation sizes h_j (1 % of p and VMR with floors 1e-7 and 1e-15,
 * 1 K, 1e-4 km^-1 for extinction).  The undisturbed forward model and all
 * n disturbed ones run as ONE batch on the GPU (n + 1 profiles, each traced
 * by every ray of obs) instead of n + 1 calls.  Like the reference, it
 * first does formod(ctl, atm, obs, aero) on the caller's data (hydrostatic
 * balance in atm->p, radiances in obs), and each disturbed profile gets
 * its own hydrostatic balance.  m, n: the matrix size, which must equal
 * jsc_obs2y's count after that forward model and jsc_atm2x's length (a
 * gsl_matrix maps as k->data, k->size1, k->size2, k->tda).  With aerosol
 * parameters in the state vector (retnn/retrr/retss, perturbed by 50 %,
 * 25 %, 10 % with floors 0.1, 0.1, 0.01) the optical properties are
 * recomputed with jsc_get_opt_prop, as formod does, and each aerosol
 * column runs the undisturbed profile as its own batch with the optical
 * properties of its disturbed parameter.  The field-of-view convolution
 * (ctl->fov) applies to every column as in formod.  For ctl->ip 2/3 (one
 * horizontally varying atmosphere per batch) each column is its own GPU
 * forward model, as in the reference. */
int jsc_kernel(ctl_t *ctl, atm_t *atm, obs_t *obs, aero_t *aero, double *k, size_t m,
               size_t n, size_t tda);

/* Number of CUDA kernels this library has launched since load. */
uint64_t jsc_launch_count(void);

/* Model: device-resident emissivity tables, Planck source tables and
 * per-channel continuum coefficients for one set of emitters, channels and
 * table files.  Built from ctl->ng/emitter/nd/nu/tblbase: reads
 * <tblbase>_<nu>_<emitter>.bin (or .tab) like read_tbl
 * (src/forwardmodel.c:610-739) and <tblbase>_<nu>.filt like srcfunc_planck
 * (src/forwardmodel.c:743-786). */
typedef struct jsc_model jsc_model;
int jsc_model_create(const ctl_t *ctl, int device, jsc_model **out);
void jsc_model_destroy(jsc_model *m);

/* Device bytes held by the model's tables. */
size_t jsc_model_table_bytes(const jsc_model *m);

/* Batch: device buffers for many independent rays over many atmospheres.
 *
 * Atmospheres are 1-D profiles (ctl->ip == 1) stored ragged: profile a has
 * levels [atm_off[a], atm_off[a+1]) of z/p/t and of q[g] and k[w], where the
 * q block is laid out [ng][n_levels_total] and k [nw][n_levels_total].
 * Ray r is traced through profile ray_atm[r].  Outputs are [n_rays][nd]. */
typedef struct jsc_batch jsc_batch;

typedef struct {
  int n_atm;
  int n_levels;              /* total levels of all profiles */
  const int *atm_off;        /* [n_atm+1] */
  const double *z, *lon, *lat, *p, *t;   /* [n_levels] */
  const double *q;           /* [ng][n_levels] */
  const double *k;           /* [nw][n_levels] */
  int n_rays;
  const int *ray_atm;        /* [n_rays] */
  const double *time;        /* [n_rays] (solar geometry) */
  const double *obsz, *obslon, *obslat;  /* [n_rays] */
  const double *vpz, *vplon, *vplat;     /* [n_rays] */
} jsc_batch_input;

typedef struct {
  double *rad;               /* [n_rays][nd] */
  double *tau;               /* [n_rays][nd] */
  double *tpz, *tplon, *tplat;  /* [n_rays], may be NULL */
  int *nlos;                 /* [n_rays] LOS points per ray, may be NULL */
} jsc_batch_output;

/* Allocate device buffers for up to max_atm profiles, max_levels levels and
 * max_rays rays (max_seg: LOS points over all rays; 0 picks a bound). */
int jsc_batch_create(jsc_model *m, const ctl_t *ctl, int max_atm,
                     int max_levels, int max_rays, int64_t max_seg,
                     jsc_batch **out);
void jsc_batch_destroy(jsc_batch *b);

/* Copy a batch's inputs from host memory to the device on stream (a
 * cudaStream_t passed as void*, NULL = default stream).  The host arrays may
 * be reused once the stream has passed this point. */
int jsc_batch_upload(jsc_batch *b, const jsc_batch_input *in, void *stream);

/* Run the forward model on the uploaded batch: hydrostatic balance (when
 * ctl->hydz >= 0), ray tracing, EGA + continua + Planck + radiative
 * transfer, all on the device, asynchronously on stream. */
int jsc_batch_run(jsc_batch *b, void *stream);

/* Copy results to host memory (waits for the stream). */
int jsc_batch_download(jsc_batch *b, const jsc_batch_output *out, void *stream);

/* upload + run + download in one call. */
int jsc_formod_batch(jsc_model *m, const ctl_t *ctl, const jsc_batch_input *in,
                     const jsc_batch_output *out, void *stream);

/* jsc_formod_batch without any device or host allocation.  No counterpart
 * in the reference: its formod (src/forwardmodel.c:15-116) keeps the line
 * of sight in a heap-allocated los_t; this entry point exists for callers
 * that must not allocate device memory while they run the forward model
 * (see below).
 *
 * Same arguments, same clear-air kernels and launch variant, same results
 * as jsc_formod_batch; host inputs and outputs as there.  Every per-call
 * device buffer (inputs, hydrostatic pressures, LOS records, outputs) is
 * carved from one static device array of JSC_NOALLOC_SCRATCH_BYTES per
 * device, so the call neither allocates nor frees (jsc_formod_batch
 * allocates and frees a whole batch per call, and cudaFree waits for the
 * whole device).  The model (its tables) must exist already.
 *
 * Limits: ctl->sca_n must be 0 (clear air); the inputs, outputs and
 * (12 + nw + ng) doubles per LOS point must fit the scratch, e.g.
 * about 390,000 LOS points for 8 emitters and one window.  A larger input
 * returns JSC_ERR_ARG with the sizes in jsc_last_error_message(), before
 * any LOS record is written.
 *
 * Set-up: the first call on a device looks up the scratch's device address
 * (cudaGetSymbolAddress, with the model's device current) and caches it;
 * make that first call before any stream capture on the device.
 *
 * Concurrency: the scratch is one per device, so two calls whose GPU work
 * overlaps would race on it.  The library holds a per-device lock for the
 * whole call and every call waits for its stream before it returns, so
 * calls from several host threads run one after another; a call that fails
 * after queueing GPU work waits for its stream before it releases the lock. */
#define JSC_NOALLOC_SCRATCH_BYTES (64u << 20)
int jsc_formod_batch_noalloc(jsc_model *m, const ctl_t *ctl,
                             const jsc_batch_input *in,
                             const jsc_batch_output *out, void *stream);

/* Per-kernel timing of the last jsc_batch_run (CUDA events on its stream).
 * kernel: "hydrostatic", "raytrace", "scatter" (scattering sources: the
 * secondary and solar pencils and the source integrals, or the surrogate
 * path), "surrogate" (the network's inference inside it), "continua" (the
 * lane variants' pre-pass), "ega_rt".  Returns milliseconds, or a
 * negative value when timing is off or the kernel did not run. */
void jsc_batch_set_timing(jsc_batch *b, int on);
double jsc_batch_kernel_ms(const jsc_batch *b, const char *kernel);

/* Launch autotuner: runs the batch once, then times every launch variant
 * of the EGA/radiative-transfer kernel (threads per block x register
 * budget) on it and keeps the fastest for later runs of this batch.
 * jsc_batch_variant reports the choice. */
int jsc_batch_autotune(jsc_batch *b, void *stream);
int jsc_batch_variant(const jsc_batch *b, int *variant, int *block, int *min_blocks);

/* Fixed-capacity runs (on != 0): jsc_batch_run then never reads back from
 * the device (LOS buffers hold the capacity given at jsc_batch_create, a
 * longer line of sight sets JSC_ERR_NLOS in the status), so upload + run +
 * download can be captured into a CUDA graph.  Covers clear air, aerosol
 * extinction (ctl->sca_mult = 0) and single scattering (ctl->sca_mult = 1,
 * ctl->ip = 1, no surrogate): there the scattering points are counted and
 * listed on the device, and a fixed number of rounds of secondary and solar
 * pencils (null pencils past the device count) run from a point list of
 * the capacity jsc_batch_set_fixed_points sets (default 40 per ray); more
 * points than that set JSC_ERR_QUEUE.  With scattering, call
 * jsc_batch_set_aero and jsc_batch_set_nalpha first: switching on
 * allocates everything the runs use (room for 144 LOS points per
 * secondary pencil and 256 per solar pencil of a round, on average). */
int jsc_batch_set_fixed(jsc_batch *b, int on);

/* Scattering-point capacity of a fixed-capacity single-scattering batch
 * (0: 40 per ray); takes effect at the next jsc_batch_set_fixed(b, 1). */
int jsc_batch_set_fixed_points(jsc_batch *b, int64_t max_points);

/* Enqueue the result copies (and the device status word) without waiting;
 * jsc_batch_async_status maps the status once the stream has passed them.
 * Requires fixed-capacity mode; host buffers should be pinned. */
int jsc_batch_download_async(jsc_batch *b, const jsc_batch_output *out, void *stream);
int jsc_batch_async_status(const jsc_batch *b);

/* Capture upload(in) + run + download_async(out) of a fixed-capacity batch
 * on stream (not the default stream) into a CUDA graph; in/out must point
 * to pinned host arrays, which later launches read and write again.
 * jsc_batch_graph_launch re-checks the inputs those arrays hold (profile
 * offsets and ray profiles, as jsc_batch_upload) and replays the graph;
 * synchronise the stream, then read the outputs and
 * jsc_batch_async_status. */
int jsc_batch_graph_capture(jsc_batch *b, const jsc_batch_input *in,
                            const jsc_batch_output *out, void *stream);
int jsc_batch_graph_launch(jsc_batch *b, void *stream);

/* Select the EGA launch variant by hand (-1: the default, variant 17, or
 * the lane variant 13 above 16 emitters).  Variants 0-8
 * run a thread per (ray, channel) with every emitter's path state; 9-13 a
 * lane per (ray, channel, emitter) after a separate continuum/Planck pass;
 * 14-20 (up to 16 emitters) lanes over a tile of 32 rays sorted by
 * geometry, a warp per emitter, after the same pass.  All variants compute
 * the same operations in the same order. */
int jsc_batch_set_variant(jsc_batch *b, int variant);
double jsc_batch_variant_ms(const jsc_batch *b, int variant);

/* Aerosol/cloud layers and optical properties for runs with ctl->sca_n > 0
 * (the aero_t that read_aero + get_opt_prop fill, src/scatter.c:330,583). */
int jsc_batch_set_aero(jsc_batch *b, const aero_t *aero);

/* Secondary pencils per scattering point of the thermal scattering source
 * (srcfunc_sca_1d, src/scatter.c:666-807, which casts 28).  nalpha: an even
 * count from 10 to 28; the zenith angles follow the reference's
 * construction (0, a Fibonacci-spaced fan, 83..90 degrees in 1-degree
 * steps, the mirrored fan, 180 degrees) with fewer fan steps.  Applies to
 * every scattering order of the batch's later runs. */
int jsc_batch_set_nalpha(jsc_batch *b, int nalpha);

/* Scattering sources at n given points through the batch's uploaded
 * profiles (the jsc_srcfunc_sca computation on a batch created with
 * ctl->sca_n > 0 and ctl->sca_mult >= 1, after jsc_batch_set_aero and
 * jsc_batch_upload; hydrostatic balance when ctl->hydz >= 0): x, dx [n][3],
 * layer [n], time [n], prof [n] (the profile of each point; NULL: 0) in
 * host memory, src [n][nd] out.  The source's order is the batch's
 * scattering depth; waits for the stream. */
int jsc_batch_scatter_points(jsc_batch *b, int n, const double *x, const double *dx,
                             const int *layer, const double *time, const int *prof,
                             double *src, void *stream);

/* Secondary pencils per scattering point for one scattering order only:
 * the points whose source srcfunc_sca computes with scattering = depth
 * (depth = ctl->sca_mult for this batch's own points, one less for the
 * points of its secondary pencils, and so on) cast nalpha pencils (even,
 * 10..28, angles as in jsc_batch_set_nalpha); other orders keep the
 * batch's count.  jsc_batch_set_nalpha resets every order to its count. */
int jsc_batch_set_nalpha_depth(jsc_batch *b, int depth, int nalpha);

/* Device waits.  The multi-block prefix scans that place LOS points and
 * scattering points (one pass, tiles waiting on their predecessors) poll an
 * unpublished predecessor at most `polls` times (0: the default, about
 * 4 M polls of at least 64 ns); a wait that runs out sets the run's status
 * to JSC_ERR_WATCHDOG and the device stays usable. */
int jsc_batch_set_wait_budget(jsc_batch *b, unsigned polls);

/* Self-test of the device-wait watchdog on `device`: the prefix scan of n
 * (1..2^26) counts with a wait budget of `budget` polls (0: default),
 * checked on the host.  stall >= 0 makes that tile never publish its sum
 * (a flag nothing sets), so its successor's wait must run out.  Returns
 * JSC_OK (scan correct), JSC_ERR_WATCHDOG (a wait gave up) or an error. */
int jsc_scan_selftest(int device, int n, unsigned budget, int stall);

/* Per-(ray, channel) checksum of every emissivity-table index the EGA
 * interpolation selected in the last run, for parity checks against the
 * reference's indices.  Per emitter g, D_g folds d = d*1000003 + v over the
 * LOS points with a full interpolation: the (p, T) bracket code
 * ipr*961 + it0*31 + it1 and then, for the (p, T) nodes (ipr,it0),
 * (ipr,it0+1), (ipr+1,it1), (ipr+1,it1+1), the interval found for the
 * path emissivity (intpol_tbl_u) and the one found for the extended column
 * (intpol_tbl_eps); the checksum folds D_0, D_1, ... the same way.  Enable
 * before jsc_batch_run (the run keeps the selected launch variant, which
 * computes its digests like every other); out is [n_rays][nd]. */
int jsc_batch_set_digest(jsc_batch *b, int on);
int jsc_batch_index_digest(jsc_batch *b, uint64_t *out);

/* Work counters of the last run: total LOS points, and the number of
 * (point, channel, emitter) EGA interpolations actually evaluated. */
int jsc_batch_counters(const jsc_batch *b, int64_t *n_points,
                       int64_t *n_ega);

/* ------------------------------------------------------------------------
 * Scattering-source surrogate (no counterpart in the reference: it stands
 * in for srcfunc_sca, src/scatter.c:643-1041, at the scattering points of
 * a batch).  A 4-layer MLP, width 128, tanh, maps 8 features of a
 * scattering point (altitude, cosine of the LOS chord's zenith angle,
 * temperature, log pressure, cosine of the solar zenith angle, cosine of
 * the solar scattering angle, layer index, solar elevation above the
 * geometric horizon) to the log of the scattering
 * source of each channel.  Trained on the GPU (FP32 forward/backward, Adam)
 * on samples of the plain source; inference runs BF16 weights on the
 * tensor cores with FP32 accumulation.
 * ------------------------------------------------------------------------ */
typedef struct jsc_surrogate jsc_surrogate;

/* A network with nd (1..64) outputs and seeded initial weights. */
int jsc_surrogate_create(int nd, int device, uint64_t seed, jsc_surrogate **out);
void jsc_surrogate_destroy(jsc_surrogate *s);

/* Parameters as one FP32 vector: W0 [128][8], b0 [128], W1 [128][128], b1,
 * W2 [128][128], b2, W3 [nd][128], b3 [nd]. */
int jsc_surrogate_param_count(const jsc_surrogate *s);
int jsc_surrogate_get_params(const jsc_surrogate *s, float *out);
int jsc_surrogate_set_params(jsc_surrogate *s, const float *in);

/* Standardisation set by jsc_surrogate_train: the network sees features
 * (X - xm) / xs (8 each) and predicts (log S - ym) / ys (nd each).  Arrays
 * may be NULL. */
int jsc_surrogate_get_scaling(const jsc_surrogate *s, float *xm, float *xs, float *ym,
                              float *ys);

/* Loss (mean over the n rows of the squared error summed over outputs) and
 * its gradient with respect to every parameter (layout of get_params), for
 * network inputs x [n][8] and targets t [n][nd] as given (no
 * standardisation); the FP32 training kernels. */
int jsc_surrogate_loss_grad(jsc_surrogate *s, const float *x, const float *t, int n,
                            float *loss, float *grads);

/* Train on n samples: raw features X [n][8] (as jsc_batch_scatter_samples
 * returns them) and plain sources src [n][nd].  Standardises features and
 * log sources, records the feature envelope, runs epochs of Adam on
 * shuffled minibatches with a cosine-decayed learning rate; loss_per_epoch
 * (may be NULL) receives the last minibatch loss of each epoch. */
int jsc_surrogate_train(jsc_surrogate *s, const float *X, const double *src, int64_t n,
                        int epochs, int batch, float lr, uint64_t seed,
                        float *loss_per_epoch);

/* Sources [n][nd] of n raw feature rows. */
int jsc_surrogate_predict(jsc_surrogate *s, const float *feat, int n, double *src);

/* Inference path: 1 (default) tcgen05 (BF16 operands in shared memory,
 * FP32 accumulators in tensor memory, 128 points per tile), 0 BF16
 * mma.sync.  Both use the same rounded weights. */
int jsc_surrogate_set_tensor_path(jsc_surrogate *s, int tcgen05);

/* Features and plain scattering sources of the last run's scattering
 * points (training data); n receives the point count, arrays may be NULL
 * to query it. */
int jsc_batch_scatter_samples(jsc_batch *b, float *feat, double *src, int64_t max, int64_t *n);

/* Use the surrogate (NULL: never) for the batch's scattering sources.
 * Points whose features leave the training envelope take the plain path;
 * every check_stride-th point inside it (0: none) is computed both ways,
 * and if for one of them omega * |S_surrogate - S_plain| / S_plain exceeds
 * tol_rel the chunk of points is recomputed with the plain path.  omega = the
 * layer's single-scattering albedo beta_s / beta_e bounds the weight of the
 * scattering source in the segment source (src/forwardmodel.c:344-349), so
 * the measure bounds the relative error of the segment source. */
int jsc_batch_set_surrogate(jsc_batch *b, jsc_surrogate *s, double tol_rel, int check_stride);

/* A surrogate for the points of one scattering order (1 .. ctl->sca_mult):
 * depth = ctl->sca_mult is jsc_batch_set_surrogate; a lower depth
 * replaces the sources at the scattering points of the batch's secondary
 * pencils of that order (for SCA_MULT = 2 and depth 1: the order-1 sources
 * along the order-1 pencils, the bulk of the cost, while the order-2
 * sources keep the plain integral over their pencils), with the same
 * envelope, sampled check and fallback, except that the check of a lower
 * order bounds the MEAN of omega |dS| / S over its checked (point,
 * channel) pairs: those sources reach the radiance only through the
 * pencil integrals of the order above, never point by point. */
int jsc_batch_set_surrogate_depth(jsc_batch *b, int depth, jsc_surrogate *s, double tol_rel,
                                  int check_stride);

/* jsc_batch_scatter_samples and jsc_batch_surrogate_stats of the batch
 * generation at scattering depth `depth` in the last run (for a lower
 * depth: the secondary-pencil batch; its samples are those of the last
 * chunk of points it ran, its statistics add up over all its chunks). */
int jsc_batch_scatter_samples_depth(jsc_batch *b, int depth, float *feat, double *src,
                                    int64_t max, int64_t *n);
int jsc_batch_surrogate_stats_depth(const jsc_batch *b, int depth, int64_t *points,
                                    int64_t *fallback, int64_t *checked, double *max_rel_err,
                                    double *mean_rel_err, int *used);

/* Surrogate counts of the last jsc_batch_run, summed over its chunks of
 * scattering points: points, fallbacks, checked points, largest relative
 * deviation found by the check, and whether every chunk used the
 * surrogate's sources (0 after any rejection); the deviation is the
 * albedo-weighted one of jsc_batch_set_surrogate. */
int jsc_batch_surrogate_stats(const jsc_batch *b, int64_t *points, int64_t *fallback,
                              int64_t *checked, double *max_rel_err, int *used);

#ifdef __cplusplus
}
#endif

#endif /* JURASSIC_B200_H */
